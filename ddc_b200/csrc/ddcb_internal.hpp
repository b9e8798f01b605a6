// ddcb_internal.hpp -- host-side plan objects and the kernel parameter blocks.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ddcb.h"
#include "bspline_math.cuh"
#include "eval_device.cuh"

namespace ddcb {

// An error carrying a ddcb_status across the C++ layers up to the C-ABI boundary.
struct Error : std::runtime_error
{
    ddcb_status status;
    Error(ddcb_status s, std::string const& msg) : std::runtime_error(msg), status(s) {}
};

#define DDCB_CUDA_CHECK(expr)                                                                      \
    do {                                                                                           \
        cudaError_t const e_ = (expr);                                                             \
        if (e_ != cudaSuccess)                                                                     \
            throw ::ddcb::Error(DDCB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Strided batched array view: element (i, b) at base[i*stride + (b/inner)*outer_stride + b%inner].
struct Lines
{
    int64_t n, stride, inner, outer, outer_stride;
    int64_t nlines() const { return inner * outer; }
};

inline Lines to_lines(ddcb_lines const& l) { return Lines {l.n, l.stride, l.inner, l.outer, l.outer_stride}; }

// Whether lines (2i, 2i+1) of a layout sit side by side at 16-byte aligned addresses, so a tile
// can move two lines per 16-byte copy.
inline bool line_pairs_aligned(const void* base, Lines const& L)
{
    return (reinterpret_cast<uintptr_t>(base) % 16 == 0) && L.stride % 2 == 0 && L.inner % 2 == 0
           && (L.outer <= 1 || L.outer_stride % 2 == 0);
}

// Device-side description of the banded solve of one builder (all pointers are device pointers).
//
// The system A (size n) is split as [[Q, g],[l, S0]] with a border of k rows/cols (periodic corner
// coupling); Q (size m = n - k) is factored P Q = L U with partial pivoting. L has kl
// sub-diagonals, U has ku super-diagonals (after pivoting fill-in). Each line is solved by
// NC chunk threads (three-phase chunked sweeps with carries, see build_kernels.cu).
struct SolveTables
{
    int n, m, k;
    int kl, ku;
    int pivot;       // 1 if any row interchange happened
    int nchunk;      // chunks per line used by the sweeps
    int chunk_len;   // chunks [0, chunk_split) have this (odd) length, the later ones two rows
    int chunk_split; // more; the last chunk ends at row m
    int nscan;       // steps of the log-depth carry scan: ceil(log2(nchunk))
    int nscan_f, nscan_b; // steps the forward / backward scans run: the transfers of later steps
                          // are below 2^-60 in every entry, so they change no carry
    int cj0, cj1, cshift; // rows [cj0, cj1) of Lf / piv / Uf are identical and stored once (at
                          // cj0); later rows move up by cshift = cj1 - cj0 - 1 (0: no run)
    int il;              // 1: Lf / piv / Uf interleaved by chunk (factor_base); 0: row-major, compressed
    const double* Lf;    // per row j, kl entries: multiplier t-1 of row j+t at step j
    const int8_t* piv;   // per row j: pivot row offset at step j (ipiv[j] - j)
    const double* Uf;    // per row j, ku+1 entries: [1/U_jj, U_j,j+1 .. U_j,j+ku]
    const double* PhiF;  // transfer over chunks c-2^k+1..c (forward), kl x kl, at scan_index
    const double* PhiB;  // transfer over chunks c..c+2^k-1 (backward), ku x ku, at scan_index
    // border (k > 0)
    int lam_nnz;
    const int* lam_row;   // k+1 row pointers into lam_col / lam_val
    const int* lam_col;
    const double* lam_val;
    const double* Sinv;  // k x k inverse of the Schur complement S0 - l Q^-1 g
    int qg_lo, qg_hi;    // rows [0, qg_lo) and [m - qg_hi, m) of Q^-1 g are kept (rest < 1e-19)
    const double* Qg;    // (qg_lo + qg_hi) x k
    // FP32 copies of the factor tables (the FP32 solves of the refinement mode)
    struct F32
    {
        const float *Lf, *Uf, *PhiF, *PhiB, *lam_val, *Sinv, *Qg;
    } f32;
    // the system matrix itself in the kernel's row / column order, CSR (FP64 residuals)
    const int* a_row;    // n+1
    const int* a_col;
    const double* a_val;
    // refinement checks: an estimate of cond_inf(A) = ||A||_inf ||A^-1||_inf (Higham's 1-norm
    // estimator for the inverse, on the host) and the builder's device status word (bit 0: a
    // refined solve missed its bound)
    double cond_est;
    double refine_tol;
    unsigned* status;
};

// Where the factor entries of row j live in the uploaded tables. Row-major tables (il = 0) store a
// row's `width` entries together, with the steady run [cj0, cj1) stored once. Interleaved tables
// (il = 1, meshes without a steady run) store entry q of step s of every chunk side by side, at
// (s * width + q) * nchunk + c, so the chunks a warp sweeps in step read one contiguous segment.
// Row j is step j - a of the chunk c that starts at row a. Entry q is at base + q * factor_stride.
DDCB_HD int factor_crow(SolveTables const& t, int j)
{
    return j < t.cj0 ? j : (j < t.cj1 ? t.cj0 : j - t.cshift);
}
DDCB_HD int factor_base(SolveTables const& t, int j, int a, int c, int width)
{
    return t.il ? ((j - a) * width) * t.nchunk + c : factor_crow(t, j) * width;
}
DDCB_HD int factor_stride(SolveTables const& t) { return t.il ? t.nchunk : 1; }
DDCB_HD int piv_index(SolveTables const& t, int j, int a, int c) { return t.il ? (j - a) * t.nchunk + c : factor_crow(t, j); }
// Entry e (row-major in the K x K matrix) of the transfer product of scan step k and chunk c.
DDCB_HD int scan_index(SolveTables const& t, int k, int e, int c, int K) { return (k * K * K + e) * t.nchunk + c; }

// How the right-hand side rows are gathered from the inputs and how the coefficients are placed.
struct RhsMap
{
    int nbe_lo, nbe_hi;   // Hermite rows at each end
    int nbv_lo, nbv_hi;   // of which read from the derivative inputs (0 for homogeneous Hermite)
    int npoints;          // interpolation values
    int offset;           // periodic column rotation (spline_builder.hpp:619-658)
    int lrot;             // tile row r holds right-hand side row (r + lrot) mod n
    int srot;             // output row o (o < n) is tile row (o - srot) mod n; rows >= n repeat
    int size;             // coefficient rows (nbasis + degree)
    int periodic;
    double dxpow_lo[8];   // dx^(i+odd) for the Hermite rows
    double dxpow_hi[8];
};

struct Basis
{
    BasisDesc desc {};          // desc.knots points at host knots
    std::vector<double> knots;  // non-uniform knots (host)
    int device = -1;
    double* d_knots = nullptr;  // device copy of knots
    BasisDesc device_desc() const
    {
        BasisDesc d = desc;
        d.knots = d_knots;
        return d;
    }
    long nbasis() const { return desc.ncells + (desc.periodic ? 0 : desc.degree); }
    long size() const { return desc.ncells + desc.degree; }
};

struct Builder
{
    Basis basis;            // own copy of the basis (knots uploaded for this builder's device)
    int lo = 0, hi = 0;
    int nbe_lo = 0, nbe_hi = 0, nbv_lo = 0, nbv_hi = 0, odd = 0;
    int offset = 0;
    int rrot = 0, crot = 0;  // rotation of rows / columns into the kernel's order (boundary blocks last)
    double dx = 0.0;
    long n = 0;             // nbasis
    std::vector<double> points;
    std::vector<double> A;  // assembled dense matrix (n x n), kept for the adjoint / checks
    int precision = DDCB_FP64;
    int refine_rounds = 2;
    double refine_tolerance = 1e-12; // bound on ||A^-1|| |b - A x| / |x| after the last round
    int device = -1;
    int tile_lines = 8;     // lines per CTA
    int nchunk_req = 64;    // requested chunks per line (64: fastest on 1000-row lines, large and small batches)
    // host copies of the solve tables (for quadrature / transposed host solves)
    int k = 0, m = 0, kl = 0, ku = 0, pivot = 0;
    std::vector<double> lu_band;   // factored Q
    std::vector<int> ipiv;
    SolveTables tables {};         // device pointers
    SolveTables tables_t {};       // tables of A^T (adjoint)
    void* d_block = nullptr;       // one allocation holding every device table
    size_t d_block_bytes = 0;
    double* d_quad = nullptr;      // quadrature weights (n, reference row order, Hermite rows scaled
                                   // by dx^k), computed on the device at creation; inside d_block
    double* d_quad_scratch = nullptr; // n doubles of d_block for that computation, then size() more
    double* d_iweights = nullptr;  // integration weights of the interpolating spline: [values (npoints),
                                   // lower derivatives (nbv_lo), upper derivatives (nbv_hi)]
    double* d_points = nullptr;    // the interpolation points on the device (inside d_block)
    unsigned* d_status = nullptr;  // device status word (inside d_block): bit 0 = not converged
    double cond_est = 0.0;         // estimate of cond_inf(A) = ||A||_inf ||A^-1||_inf
    RhsMap rhs {};
    std::string structure;
    void* host_private = nullptr;  // host factorisation (plan.cpp)
};

struct Evaluator
{
    Basis basis;
    int ex_lo = DDCB_EXTRAP_NULL, ex_hi = DDCB_EXTRAP_NULL;
    int device = -1;
    EvalBasis eb {};               // device view: knots, knot-span inverses, cell lookup table
    double* d_integrals = nullptr; // integrals of the B-splines (size entries), inside d_block
    void* d_block = nullptr;
    std::vector<double> integrals;
};

Evaluator* create_evaluator(Basis const& basis, int ex_lo, int ex_hi);
void destroy_evaluator(Evaluator* e);

// plan.cpp
void make_uniform_basis(Basis& b, int degree, bool periodic, double rmin, double rmax, long ncells);
void make_non_uniform_basis(Basis& b, int degree, bool periodic, double const* breaks, long nbreaks);
void upload_basis(Basis& b, int device);
void free_basis(Basis& b);
std::vector<double> greville_points(Basis const& b, int lo, int hi);
void basis_integrals(Basis const& b, double* out);
Builder* create_builder(Basis const& basis, double const* pts, long npts, int lo, int hi, ddcb_builder_options const* opts);
// host part of create_builder (no CUDA call) and the device upload it is followed by
Builder* create_builder_host(Basis const& basis, double const* pts, long npts, int lo, int hi, ddcb_builder_options const* opts);
void upload_builder(Builder* b);
double emulate_device_solve(Builder const& b, double const* rhs, bool transpose);
double emulate_build(Builder const& b, double const* vals, double const* dlo, double const* dhi);
void destroy_builder(Builder* b);
// Most dimensions of a tensor-product evaluation (SplineEvaluatorND).
constexpr int kMaxDims = 6;

// quadrature.cu: weights by the device transposed solve (d_qk: n doubles of scratch), and the
// integral of the interpolating spline of every line straight from its samples.
void compute_device_quadrature(Builder& b, double* d_qk, double* d_q);
void launch_integrate_samples(Builder const& b, double* out, int64_t out_outer_stride, double const* vals, Lines const& lv,
                              double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi, cudaStream_t s);

// build_kernels.cu
void launch_build(Builder const& b, double* coefs, Lines const& lc, double const* vals, Lines const& lv,
                  double const* dlo, Lines const& llo, double const* dhi, Lines const& lhi, cudaStream_t s);
void launch_solve_multirhs(Builder const& b, double* rhs, long ld, long nrhs, bool transpose, cudaStream_t s);
// Builder then evaluator on the same lines; returns true when the single fused kernel ran.
bool launch_build_eval(Builder const& b, Evaluator const& e, int order, double* coefs, Lines const& lc,
                       double const* vals, Lines const& lv, double const* dlo, Lines const& llo, double const* dhi,
                       Lines const& lhi, double const* coords, Lines const& lx, double* out, Lines const& lo, cudaStream_t s);

// One semi-Lagrangian advection step (examples/characteristics_advection.cpp:243-259): build the
// lines' splines, evaluate each at the feet pts[q] - dt * v(b) of the interpolation points, with
// v(b) = velocity[b / v_div] or v_const. coefs may be NULL (not kept). Returns true when one
// fused kernel ran (uniform bases); otherwise a build, a feet kernel and an evaluation run with
// stream-ordered scratch.
bool launch_advect(Builder const& b, Evaluator const& e, double dt, double const* velocity, double v_const, int64_t v_div,
                   double* out, Lines const& lo, double const* vals, Lines const& lv, double const* dlo, Lines const& llo,
                   double const* dhi, Lines const& lhi, double* coefs, Lines const& lc, cudaStream_t s);

// adjoint_kernels.cu
void launch_build_adjoint(Builder const& b, double const* gc, Lines const& lgc, double* gv, Lines const& lgv,
                          double* gdlo, Lines const& lglo, double* gdhi, Lines const& lghi, cudaStream_t s);
void launch_eval_adjoint(Evaluator const& e, int order, double const* coords, Lines const& lx, double const* coefs,
                         Lines const& lc, double const* gy, Lines const& lgy, double* gc, Lines const& lgc, double* gx,
                         Lines const& lgx, cudaStream_t s);
// Returns whether the single fused kernel ran (else the two kernels above did, through a
// stream-ordered cotangent buffer).
bool launch_build_eval_adjoint(Builder const& b, Evaluator const& e, int order, double const* coords, Lines const& lx,
                               double const* coefs, Lines const& lc, double const* gy, Lines const& lgy, double* gv,
                               Lines const& lgv, double* gdlo, Lines const& lglo, double* gdhi, Lines const& lghi,
                               double* gx, Lines const& lgx, cudaStream_t s);

// host_pipeline.cu: build + evaluate on host buffers, batch slices pipelined over three streams.
// Host layouts have outer == 1 (rows of the batch, any row stride >= inner) or inner == 1 with unit
// stride (one contiguous line per batch index).
struct HostArrays
{
    const double* vals = nullptr;
    Lines lv {};
    const double* dlo = nullptr; // NULL when the lower closure reads no derivative
    Lines llo {};
    const double* dhi = nullptr;
    Lines lhi {};
    const double* coords = nullptr;
    Lines lx {};
    double* out = nullptr;
    Lines lo {};
    double* coefs = nullptr; // optional copy of the coefficients
    Lines lc {};
};
struct HostPipeline
{
    Builder const* b = nullptr;
    Evaluator const* e = nullptr;
    int order = 0;
    int64_t m = 0;     // evaluation points per line
    int64_t slice = 0; // lines per slice
    int device = 0;
    void* d_block = nullptr;
    double* buf[2][6] = {}; // per buffer set: vals, derivs_lo, derivs_hi, coords, out, coefs
    cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
    cudaEvent_t ev_start = nullptr, in_done[2] = {}, comp_done[2] = {}, out_done[2] = {};
};
HostPipeline* create_host_pipeline(Builder const& b, Evaluator const& e, int order, int64_t m, int64_t slice);
void destroy_host_pipeline(HostPipeline* p);
void run_host_pipeline(HostPipeline& p, int64_t nbatch, HostArrays const& h, cudaStream_t user);

// uneven_batch.cu
struct UnevenBatch;
UnevenBatch* create_uneven_batch(Builder const* const* builders, Evaluator const* const* evals, int64_t const* nevals,
                                 int64_t count);
void destroy_uneven_batch(UnevenBatch* b);
void uneven_offsets(UnevenBatch const& b, int64_t* vals, int64_t* dlo, int64_t* dhi, int64_t* coefs, int64_t* evals);
void uneven_info(UnevenBatch const& b, int64_t* totals, int* schedule, double* tuned_us);
void run_uneven_batch(UnevenBatch& b, double const* vals, double const* dlo, double const* dhi, double* coefs,
                      double const* coords, double* out, cudaStream_t s);
void tune_uneven_batch(UnevenBatch& b, double const* vals, double const* dlo, double const* dhi, double* coefs,
                       double const* coords, double* out, int reps, cudaStream_t s);

// tensor2d.cu
// A second stream of the calling host thread on the current device, with the two events of a
// fork and a join: the 2D and 3D builds run their short derivative-slab passes there, beside the
// long value pass, and join before the passes that read them. Kept per host thread (the calls of
// one thread are ordered), created on first use and kept until the thread ends.
struct SideStream
{
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
SideStream& side_stream_for_current_device();
size_t build2d_workspace_bytes(Builder const& b1, Builder const& b2, int64_t nbatch);
void launch_build2d(Builder const& b1, Builder const& b2, double* coefs, double const* vals, double const* dmin1,
                    double const* dmax1, double const* dmin2, double const* dmax2, double const* m11, double const* m21,
                    double const* m12, double const* m22, int64_t B, double* ws, cudaStream_t s, int64_t max_group = 0,
                    bool overlap_slabs = false);
void launch_eval2d(Evaluator const& e1, Evaluator const& e2, int o1, int o2, double* out, double const* coords,
                   double const* coefs, int64_t m, int64_t B, cudaStream_t s);
void launch_integrate2d(Evaluator const& e1, Evaluator const& e2, double* out, double const* coefs, int64_t B, cudaStream_t s);

// tensornd.cu: 3D builder (inputs: 27 arrays, index k1 + 3 k2 + 9 k3 with k = 0 values, 1 lower,
// 2 upper derivatives along that dimension) and the N-dimensional evaluator / integrator.
size_t build3d_workspace_bytes(Builder const& b1, Builder const& b2, Builder const& b3, int64_t B);
void launch_build3d(Builder const& b1, Builder const& b2, Builder const& b3, double* coefs, double const* const* inputs,
                    int64_t B, double* ws, cudaStream_t s);
void launch_evalnd(Evaluator const* const* e, int ndims, int const* orders, double* out, double const* coords,
                   double const* coefs, int64_t m, int64_t B, cudaStream_t s);
void launch_integratend(Evaluator const* const* e, int ndims, double* out, double const* coefs, int64_t B, cudaStream_t s);
size_t build2d_static_scratch_bytes();
void launch_build2d_static(Builder const& b1, Builder const& b2, double* coefs, double const* vals, double const* dmin1,
                           double const* dmax1, double const* dmin2, double const* dmax2, double const* m11,
                           double const* m21, double const* m12, double const* m22, int64_t B, cudaStream_t s);

// eval_kernels.cu
void launch_eval(Evaluator const& e, int order, double* out, Lines const& lo, double const* coords, Lines const& lx,
                 double const* coefs, Lines const& lc, cudaStream_t s);
void launch_integrate(Evaluator const& e, double* out, int64_t out_stride, double const* coefs, Lines const& lc,
                      cudaStream_t s);

} // namespace ddcb
