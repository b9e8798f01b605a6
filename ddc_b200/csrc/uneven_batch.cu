// uneven_batch.cu -- thousands of independent 1D spline problems of different size, degree,
// closure and mesh, built and evaluated in ONE graph launch.
//
// Each problem is one line: a builder (its device factor tables) and an evaluator, with its
// samples, derivatives, coefficients, coordinates and values packed one after another in flat
// arrays. Problems are grouped by the band shape of their factors and their arithmetic (the solve
// is compiled per shape: one kernel holding every shape's solve spills registers; FP64 or FP32 with
// FP64 refinement), and by block size: under the warp schedule a problem's block has one thread
// per chunk of its plan, rounded up to a warp, so short problems (<= 32 chunks) run one warp each,
// many per SM, with barriers that cost a warp's; under the block schedule every block has
// `threads` threads. A problem is a tile of ONE line: the chunk threads sweep scalar rows (no
// empty partner line), so a problem's shared memory is its n rows plus the chunk carries.
//
// Each group gets a build kernel whose grid holds, by default, one block per problem (block b
// starts with queue position b; with a smaller grid, later problems come from a counter, in
// largest-first order by default). A block copies its problem's description into shared memory,
// gathers the right-hand side, runs the chunked tile solve of the batched builder (the chunks'
// carries chained by the log-depth scan across the block's threads) and stores the coefficients.
// Each group's evaluation kernel, which depends on that group's build kernel only, evaluates the
// group's points from the stored coefficients with 256-thread blocks over segments of 1024 points,
// so the points of a problem are spread over many threads instead of waiting on its chunk
// threads, and the short problems' evaluations overlap the long problems' builds. The build
// kernels of the groups with the longest problems get the highest stream priorities.
//
// ddcb_batch_uneven_run launches a CUDA graph holding the counter reset and the group kernels,
// which run concurrently; the graph is rebuilt only when the buffers, stream or schedule change.
// ddcb_batch_uneven_tune times the candidate schedules (warp or block schedule, block size, the
// per-SM thread budget, queue order), each as the graph it would run as, on the caller's buffers
// and keeps the fastest.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "build_device.cuh"
#include "eval_device.cuh"
#include "refine_device.cuh"

namespace ddcb {

// Band shapes of the plan's menu (plan.cpp, HostSolve::analyse), by index.
static int const kShapes[][2] = {{1, 1}, {1, 2}, {2, 2}, {3, 3}, {1, 4}, {2, 4}, {4, 4}, {3, 6}, {1, 8}, {2, 8}, {4, 8}};
static int const kNumShapes = int(sizeof(kShapes) / sizeof(kShapes[0]));

struct UnevenProblem
{
    BuildArgs args;        // data pointers hold offsets into the packed arrays (added at run time)
    int shape;             // index into kShapes
    int rounds;            // refinement rounds (FP32 solve); -1: FP64 solve
};

// What the evaluation of one problem needs.
struct UnevenEval
{
    EvalBasis eb;
    int ex_lo, ex_hi;
    int degree, uniform;
    int m;                 // evaluation points
    int64_t x_off;         // first coordinate (and output value) in the packed arrays
    int64_t coef_off;      // first coefficient in the packed array
};

struct UnevenArgs
{
    const UnevenProblem* probs;
    const int* order;      // queue order of the group's problems
    int nprob;
    int* counter;          // next queue position (reset to 0 before each launch)
    const double* vals;
    const double* dlo;
    const double* dhi;
    double* coefs;
};

// A block's share of one problem's points: kSegment points from `first` on (fewer at the end).
struct UnevenSegment
{
    int prob;
    int first;
    int64_t x;             // packed index of its first coordinate and value
};

struct UnevenEvalArgs
{
    const UnevenEval* evals;
    const UnevenSegment* segs;
    const double* coefs;
    const double* coords;
    double* out;
};

// Sweep rows unrolled per step (their factor loads issue together) and no transfer-matrix loads
// ahead of the scan barriers (registers for more resident problems): measured on the uneven
// workload of 4096 problems.
constexpr int kUnevenUnroll = 4;
constexpr bool kUnevenScanPrefetch = false;
constexpr int kEvalThreads = 256;
constexpr int kEvalPts = 4;                           // points per thread
constexpr int kSegment = kEvalThreads * kEvalPts;     // points per evaluation block

namespace {

template <int KL, int KU, bool REFINE>
__global__ void __launch_bounds__(512, 1) uneven_build_kernel(const __grid_constant__ UnevenArgs A)
{
    extern __shared__ __align__(16) double smem[];
    __shared__ UnevenProblem sp;
    __shared__ int s_next;
    // the first problem of block b is queue position b; later ones come from the counter
    for (int pass = 0;; ++pass) {
        if (pass > 0) {
            if (threadIdx.x == 0) s_next = int(gridDim.x) + atomicAdd(A.counter, 1);
            __syncthreads();
        }
        int const qi = pass > 0 ? s_next : int(blockIdx.x);
        if (qi >= A.nprob) break;
        // the problem's description into shared memory, offsets turned into pointers
        {
            const int* src = reinterpret_cast<const int*>(A.probs + A.order[qi]);
            int* dst = reinterpret_cast<int*>(&sp);
            for (int i = threadIdx.x; i < int(sizeof(UnevenProblem) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            sp.args.vals = A.vals + reinterpret_cast<intptr_t>(sp.args.vals);
            sp.args.dlo = A.dlo + reinterpret_cast<intptr_t>(sp.args.dlo);
            sp.args.dhi = A.dhi + reinterpret_cast<intptr_t>(sp.args.dhi);
            sp.args.out = A.coefs + reinterpret_cast<intptr_t>(sp.args.out);
            sp.args.nct = blockDim.x;
        }
        __syncthreads();
        // register copies of the tables: read from shared memory, their addresses would have to be
        // reloaded after every store to the tile (the compiler cannot rule out aliasing), which
        // serialises the sweeps' factor loads row by row
        if constexpr (REFINE) {
            BuildArgs const args = sp.args;
            refine_tile<1, KL, KU>(args, smem, sp.rounds);
        } else {
            gather_tile<1>(sp.args, smem);
            SolveTables const t = sp.args.t;
            solve_in_tile<1, KL, KU, double, kUnevenUnroll, kUnevenScanPrefetch>(t, 0, smem);
        }
        store_tile<1>(sp.args, smem);
        __syncthreads(); // the tile and the description are reused by the next problem
    }
}

// The thread's points of a segment (q0 + k * kEvalThreads, k < kEvalPts): coordinates loaded
// first, so the evaluations' load chains overlap.
template <int D, bool UNI>
__device__ __forceinline__ void eval_seg(UnevenEval const& e, double const* coefs, double const* xv, double* y, int live)
{
    CoefGlobal const acc {coefs + e.coef_off, 1};
#pragma unroll
    for (int k = 0; k < kEvalPts; ++k)
        if (k < live) __stcs(y + k * kEvalThreads, eval_point<D, 0, UNI>(e.eb, e.ex_lo, e.ex_hi, xv[k], acc));
}

// One block per segment of a problem's points (kEvalPts per thread); the coefficients come from
// the build kernels (the graph orders them before this kernel).
__global__ void __launch_bounds__(kEvalThreads, 4) uneven_eval_kernel(const __grid_constant__ UnevenEvalArgs A)
{
    __shared__ UnevenEval se;
    UnevenSegment const seg = A.segs[blockIdx.x];
    // the description and this thread's coordinates load together
    {
        const int* src = reinterpret_cast<const int*>(A.evals + seg.prob);
        int* dst = reinterpret_cast<int*>(&se);
        for (int i = threadIdx.x; i < int(sizeof(UnevenEval) / sizeof(int)); i += blockDim.x) dst[i] = __ldg(src + i);
    }
    double xv[kEvalPts];
    int live = 0;
    {
        int const m = __ldg(&A.evals[seg.prob].m);
#pragma unroll
        for (int k = 0; k < kEvalPts; ++k) {
            int const q = seg.first + int(threadIdx.x) + k * kEvalThreads;
            xv[k] = q < m ? __ldcs(A.coords + seg.x + threadIdx.x + k * kEvalThreads) : 0.0;
            live += q < m ? 1 : 0;
        }
    }
    __syncthreads();
    if (live == 0) return;
    double* y = A.out + seg.x + threadIdx.x;
    // a register copy, for the reason the build kernel keeps one of its tables
    UnevenEval const e = se;
    switch (e.degree * 2 + e.uniform) {
    case 2: eval_seg<1, false>(e, A.coefs, xv, y, live); break;
    case 3: eval_seg<1, true>(e, A.coefs, xv, y, live); break;
    case 4: eval_seg<2, false>(e, A.coefs, xv, y, live); break;
    case 5: eval_seg<2, true>(e, A.coefs, xv, y, live); break;
    case 6: eval_seg<3, false>(e, A.coefs, xv, y, live); break;
    case 7: eval_seg<3, true>(e, A.coefs, xv, y, live); break;
    case 8: eval_seg<4, false>(e, A.coefs, xv, y, live); break;
    case 9: eval_seg<4, true>(e, A.coefs, xv, y, live); break;
    case 10: eval_seg<5, false>(e, A.coefs, xv, y, live); break;
    default: eval_seg<5, true>(e, A.coefs, xv, y, live); break;
    }
}

using UnevenKernel = void (*)(UnevenArgs);

template <bool R>
UnevenKernel kernel_of_r(int shape)
{
    switch (shape) {
    case 0: return uneven_build_kernel<1, 1, R>;
    case 1: return uneven_build_kernel<1, 2, R>;
    case 2: return uneven_build_kernel<2, 2, R>;
    case 3: return uneven_build_kernel<3, 3, R>;
    case 4: return uneven_build_kernel<1, 4, R>;
    case 5: return uneven_build_kernel<2, 4, R>;
    case 6: return uneven_build_kernel<4, 4, R>;
    case 7: return uneven_build_kernel<3, 6, R>;
    case 8: return uneven_build_kernel<1, 8, R>;
    case 9: return uneven_build_kernel<2, 8, R>;
    default: return uneven_build_kernel<4, 8, R>;
    }
}

UnevenKernel kernel_of(int shape, bool refine) { return refine ? kernel_of_r<true>(shape) : kernel_of_r<false>(shape); }

size_t problem_smem(UnevenProblem const& p)
{
    int const kl = kShapes[p.shape][0], ku = kShapes[p.shape][1];
    return p.rounds >= 0 ? refine_smem(p.args.t, 1, kl, ku) : sizeof(double) * tile_doubles(p.args.t, 1, kl, ku);
}

// The block of a problem under the warp schedule: one thread per chunk, whole warps.
int warp_class(int nchunk) { return std::max(32, (nchunk + 31) / 32 * 32); }

} // namespace

struct UnevenBatch
{
    int device = -1;
    int64_t count = 0;
    std::vector<int64_t> vals_off, dlo_off, dhi_off, coef_off, x_off; // count + 1 prefix sums
    UnevenProblem* d_probs = nullptr;
    UnevenEval* d_evals = nullptr;
    UnevenSegment* d_segs = nullptr; // evaluation segments
    int64_t nseg = 0;
    // per group (band shape, arithmetic, warp-schedule block size): its problems in two queue
    // orders (largest-first, then natural) at d_order + 2*gfirst[g] and d_order + 2*gfirst[g] +
    // gsize[g]; its counter d_counter[g]
    std::vector<int> gshape, grefine, gclass, gfirst, gsize;
    std::vector<int64_t> gseg0, gnseg;  // the group's evaluation segments in d_segs
    std::vector<double> gcost, gmax;  // per group: total and largest problem cost
    std::vector<int> grank;           // groups ranked by their largest problem (0: the largest)
    int nrank = 1;
    std::vector<size_t> gsmem;
    int* d_order = nullptr;
    int* d_counter = nullptr;
    size_t smem = 0;
    int max_chunks = 0;
    // schedule
    int warp = 1;              // 1: blocks sized to each problem's chunks; 0: `threads` for every block
    int threads = 256;
    int blocks_per_sm = 0;     // per-SM budget in units of 256 threads (0: as many blocks as fit)
    int order = 0;             // 0 largest-first, 1 natural
    int prio = 1;              // 1: the groups' kernels get priorities by their largest problem
    double tuned_us = 0.0;
    // cached graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    UnevenArgs key {};
    const double* key_coords = nullptr;
    double* key_out = nullptr;
    cudaStream_t key_stream = nullptr;
    int key_threads = 0, key_blocks = 0, key_order = -1, key_warp = -1;
};

namespace {

int sm_count()
{
    int dev = 0, sms = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    DDCB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

// Block size of group g under the current schedule.
int group_threads(UnevenBatch const& b, int g)
{
    int const c = b.gclass[size_t(g)];
    return b.warp ? c : std::max(b.threads, c);
}

// Blocks of group g's kernel: the per-SM budget (blocks_per_sm x 256 threads; 0: as many blocks
// as fit) over the SMs, at least one, at most its problem count.
int group_blocks(UnevenBatch const& b, int g, int threads, int per_sm)
{
    UnevenKernel k = kernel_of(b.gshape[size_t(g)], b.grefine[size_t(g)] != 0);
    size_t const sm = b.gsmem[size_t(g)];
    if (sm > 48 * 1024) DDCB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    int fit = 0;
    DDCB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k, threads, sm));
    if (fit < 1) throw Error(DDCB_ERR_UNSUPPORTED, "the largest problem's tile does not fit in shared memory");
    // every group may start all its problems at once: its grid is capped by its problem count and
    // by the blocks that fit (or the budget); the groups' kernels share the GPU concurrently, and
    // blocks that do not fit yet queue behind the running ones
    int const per = per_sm > 0 ? std::min(std::max(1, per_sm * 256 / threads), fit) : fit;
    int64_t const blocks = int64_t(per) * sm_count();
    return int(std::max<int64_t>(1, std::min<int64_t>(blocks, b.gsize[size_t(g)])));
}

UnevenArgs make_args(UnevenBatch const& b, int g, int order, double const* vals, double const* dlo, double const* dhi,
                     double* coefs)
{
    UnevenArgs a {};
    a.probs = b.d_probs;
    a.order = b.d_order + 2 * b.gfirst[size_t(g)] + (order ? b.gsize[size_t(g)] : 0);
    a.nprob = b.gsize[size_t(g)];
    a.counter = b.d_counter + g;
    a.vals = vals;
    a.dlo = dlo;
    a.dhi = dhi;
    a.coefs = coefs;
    return a;
}

void drop_graph(UnevenBatch& b)
{
    if (b.exec) cudaGraphExecDestroy(b.exec);
    if (b.graph) cudaGraphDestroy(b.graph);
    b.exec = nullptr;
    b.graph = nullptr;
}

} // namespace

UnevenBatch* create_uneven_batch(Builder const* const* builders, Evaluator const* const* evals, int64_t const* nevals,
                                 int64_t count)
{
    auto* b = new UnevenBatch();
    try {
        DDCB_CUDA_CHECK(cudaGetDevice(&b->device));
        b->count = count;
        std::vector<UnevenProblem> probs(static_cast<size_t>(count));
        std::vector<UnevenEval> evs(static_cast<size_t>(count));
        std::vector<UnevenSegment> segs;
        b->vals_off.assign(size_t(count) + 1, 0);
        b->dlo_off = b->dhi_off = b->coef_off = b->x_off = b->vals_off;
        std::vector<double> cost(static_cast<size_t>(count));
        for (int64_t i = 0; i < count; ++i) {
            Builder const& bl = *builders[i];
            Evaluator const& ev = *evals[i];
            std::string const who = "problem " + std::to_string(i) + ": ";
            if (bl.device != b->device || ev.device != b->device) throw Error(DDCB_ERR_INVALID_ARGUMENT, who + "created for another device");
            if (ev.basis.desc.degree != bl.basis.desc.degree || ev.basis.desc.ncells != bl.basis.desc.ncells
                || ev.basis.desc.periodic != bl.basis.desc.periodic || ev.basis.desc.uniform != bl.basis.desc.uniform)
                throw Error(DDCB_ERR_INVALID_ARGUMENT, who + "builder and evaluator use different bases");
            if (nevals[i] < 0 || nevals[i] > (int64_t(1) << 30)) throw Error(DDCB_ERR_INVALID_ARGUMENT, who + "bad evaluation count");
            UnevenProblem& p = probs[size_t(i)];
            p.rounds = bl.precision == DDCB_FP32_REFINE ? bl.refine_rounds : -1;
            p.shape = -1;
            for (int sh = 0; sh < kNumShapes; ++sh)
                if (kShapes[sh][0] == bl.tables.kl && kShapes[sh][1] == bl.tables.ku) p.shape = sh;
            if (p.shape < 0) throw Error(DDCB_ERR_UNSUPPORTED, who + "band shape has no kernel");
            if (bl.tables.nchunk > 512) throw Error(DDCB_ERR_UNSUPPORTED, who + "more than 512 chunks per line");
            int64_t const np = int64_t(bl.points.size()), size = int64_t(bl.basis.size());
            b->vals_off[i + 1] = b->vals_off[i] + np;
            b->dlo_off[i + 1] = b->dlo_off[i] + (bl.lo == DDCB_HERMITE ? bl.nbv_lo : 0);
            b->dhi_off[i + 1] = b->dhi_off[i] + (bl.hi == DDCB_HERMITE ? bl.nbv_hi : 0);
            b->coef_off[i + 1] = b->coef_off[i] + size;
            b->x_off[i + 1] = b->x_off[i] + nevals[i];
            BuildArgs& a = p.args;
            a.t = bl.tables;
            a.r = bl.rhs;
            a.raw = 0;
            a.nlines = 1;
            // offsets into the packed arrays, turned into pointers by the kernel
            a.vals = reinterpret_cast<const double*>(intptr_t(b->vals_off[i]));
            a.dlo = reinterpret_cast<const double*>(intptr_t(b->dlo_off[i]));
            a.dhi = reinterpret_cast<const double*>(intptr_t(b->dhi_off[i]));
            a.out = reinterpret_cast<double*>(intptr_t(b->coef_off[i]));
            a.lv = Lines {np, 1, 1, 1, 0};
            a.llo = Lines {bl.nbv_lo, 1, 1, 1, 0};
            a.lhi = Lines {bl.nbv_hi, 1, 1, 1, 0};
            a.lo = Lines {size, 1, 1, 1, 0};
            a.pair16 = a.pair16_out = 0;
            a.line_base = 0; // one line per problem, its arrays already offset
            UnevenEval& e = evs[size_t(i)];
            e.eb = ev.eb;
            e.ex_lo = ev.ex_lo;
            e.ex_hi = ev.ex_hi;
            e.degree = ev.basis.desc.degree;
            e.uniform = ev.basis.desc.uniform ? 1 : 0;
            e.m = int(nevals[i]);
            e.x_off = b->x_off[i];
            e.coef_off = b->coef_off[i];
            b->max_chunks = std::max(b->max_chunks, bl.tables.nchunk);
            // a block's time on a problem: a fixed part (barriers, scans, the description) plus
            // the rows its threads step through
            cost[size_t(i)] = 64.0 + double(np) * (kShapes[p.shape][0] + kShapes[p.shape][1] + 2) / 8.0
                              ;
        }
        // groups by band shape, arithmetic and warp-schedule block size (the tile of a group is
        // sized to its largest problem); queue orders within each group
        std::vector<int> order;
        for (int sh = 0; sh < kNumShapes; ++sh) {
            for (int rf = 0; rf < 2; ++rf) {
                for (int cls = 32; cls <= 512; cls += 32) {
                    std::vector<int> members;
                    size_t smem = 0;
                    double c = 0.0, cmax = 0.0;
                    for (int64_t i = 0; i < count; ++i) {
                        UnevenProblem const& p = probs[size_t(i)];
                        if (p.shape != sh || (p.rounds >= 0) != (rf == 1) || warp_class(p.args.t.nchunk) != cls) continue;
                        members.push_back(int(i));
                        smem = std::max(smem, problem_smem(p));
                        c += cost[size_t(i)];
                        cmax = std::max(cmax, cost[size_t(i)]);
                    }
                    if (members.empty()) continue;
                    b->gshape.push_back(sh);
                    b->grefine.push_back(rf);
                    b->gclass.push_back(cls);
                    b->gfirst.push_back(int(order.size() / 2));
                    b->gsize.push_back(int(members.size()));
                    b->gcost.push_back(c);
                    b->gmax.push_back(cmax);
                    b->gsmem.push_back((smem + 15) & ~size_t(15));
                    b->smem = std::max(b->smem, b->gsmem.back());
                    std::vector<int> lpt = members;
                    std::stable_sort(lpt.begin(), lpt.end(), [&](int x, int y) { return cost[size_t(x)] > cost[size_t(y)]; });
                    order.insert(order.end(), lpt.begin(), lpt.end());
                    order.insert(order.end(), members.begin(), members.end());
                    // the group's evaluation segments, largest problems first
                    b->gseg0.push_back(int64_t(segs.size()));
                    for (int i : lpt) {
                        UnevenEval const& e = evs[size_t(i)];
                        for (int q0 = 0; q0 < e.m; q0 += kSegment) segs.push_back(UnevenSegment {i, q0, e.x_off + q0});
                    }
                    b->gnseg.push_back(int64_t(segs.size()) - b->gseg0.back());
                }
            }
        }
        if (count > 0) {
            DDCB_CUDA_CHECK(cudaMalloc(&b->d_probs, sizeof(UnevenProblem) * size_t(count)));
            DDCB_CUDA_CHECK(cudaMemcpy(b->d_probs, probs.data(), sizeof(UnevenProblem) * size_t(count), cudaMemcpyHostToDevice));
            DDCB_CUDA_CHECK(cudaMalloc(&b->d_order, sizeof(int) * order.size()));
            DDCB_CUDA_CHECK(cudaMemcpy(b->d_order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice));
            DDCB_CUDA_CHECK(cudaMalloc(&b->d_evals, sizeof(UnevenEval) * size_t(count)));
            DDCB_CUDA_CHECK(cudaMemcpy(b->d_evals, evs.data(), sizeof(UnevenEval) * size_t(count), cudaMemcpyHostToDevice));
        }
        {
            std::vector<int> idx(b->gmax.size());
            std::iota(idx.begin(), idx.end(), 0);
            std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return b->gmax[size_t(x)] > b->gmax[size_t(y)]; });
            b->grank.assign(idx.size(), 0);
            for (size_t r = 0; r < idx.size(); ++r) b->grank[size_t(idx[r])] = int(r);
            b->nrank = std::max<int>(1, int(idx.size()));
        }
        if (segs.size() >= size_t(1) << 31) throw Error(DDCB_ERR_UNSUPPORTED, "more than 2^31 evaluation segments");
        b->nseg = int64_t(segs.size());
        if (b->nseg > 0) {
            DDCB_CUDA_CHECK(cudaMalloc(&b->d_segs, sizeof(UnevenSegment) * segs.size()));
            DDCB_CUDA_CHECK(cudaMemcpy(b->d_segs, segs.data(), sizeof(UnevenSegment) * segs.size(), cudaMemcpyHostToDevice));
        }
        DDCB_CUDA_CHECK(cudaMalloc(&b->d_counter, sizeof(int) * std::max<size_t>(1, b->gshape.size())));
        b->threads = std::max(256, (b->max_chunks + 31) / 32 * 32);
        return b;
    } catch (...) {
        destroy_uneven_batch(b);
        throw;
    }
}

void destroy_uneven_batch(UnevenBatch* b)
{
    if (!b) return;
    drop_graph(*b);
    if (b->d_probs) cudaFree(b->d_probs);
    if (b->d_evals) cudaFree(b->d_evals);
    if (b->d_segs) cudaFree(b->d_segs);
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_counter) cudaFree(b->d_counter);
    delete b;
}

void uneven_offsets(UnevenBatch const& b, int64_t* vals, int64_t* dlo, int64_t* dhi, int64_t* coefs, int64_t* evals)
{
    auto copy = [&](std::vector<int64_t> const& v, int64_t* o) {
        if (o) std::copy(v.begin(), v.end(), o);
    };
    copy(b.vals_off, vals);
    copy(b.dlo_off, dlo);
    copy(b.dhi_off, dhi);
    copy(b.coef_off, coefs);
    copy(b.x_off, evals);
}

void uneven_info(UnevenBatch const& b, int64_t* totals, int* schedule, double* tuned_us)
{
    totals[0] = b.count;
    totals[1] = b.vals_off.back();
    totals[2] = b.dlo_off.back();
    totals[3] = b.dhi_off.back();
    totals[4] = b.coef_off.back();
    totals[5] = b.x_off.back();
    schedule[0] = b.threads;
    schedule[1] = b.blocks_per_sm;
    schedule[2] = b.order;
    schedule[3] = int(b.smem);
    schedule[4] = b.warp;
    *tuned_us = b.tuned_us;
}

void run_uneven_batch(UnevenBatch& b, double const* vals, double const* dlo, double const* dhi, double* coefs,
                      double const* coords, double* out, cudaStream_t s)
{
    if (b.count == 0) return;
    UnevenArgs const key = make_args(b, 0, b.order, vals, dlo, dhi, coefs);
    bool const stale = !b.exec || key.vals != b.key.vals || key.dlo != b.key.dlo || key.dhi != b.key.dhi
                       || key.coefs != b.key.coefs || coords != b.key_coords || out != b.key_out
                       || s != b.key_stream || b.threads != b.key_threads || b.blocks_per_sm != b.key_blocks
                       || b.order != b.key_order || b.warp != b.key_warp;
    if (stale) {
        drop_graph(b);
        DDCB_CUDA_CHECK(cudaGraphCreate(&b.graph, 0));
        cudaMemsetParams mp {};
        mp.dst = b.d_counter;
        mp.value = 0;
        mp.elementSize = sizeof(int);
        mp.width = b.gshape.size();
        mp.height = 1;
        mp.pitch = 0;
        cudaGraphNode_t mnode = nullptr;
        DDCB_CUDA_CHECK(cudaGraphAddMemsetNode(&mnode, b.graph, nullptr, 0, &mp));
        // the groups of the longest problems first in the block scheduler's eye: their kernels
        // are added first and get the higher priorities (the graph is instantiated to use node
        // priorities), so their blocks are not queued behind the short problems'
        int least = 0, greatest = 0;
        DDCB_CUDA_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        int const ng = int(b.gshape.size());
        std::vector<int> by_rank(size_t(ng), 0);
        for (int g = 0; g < ng; ++g) by_rank[size_t(b.grank[size_t(g)])] = g;
        std::vector<cudaGraphNode_t> built(size_t(ng), nullptr);
        for (int g : by_rank) {
            UnevenArgs args = make_args(b, g, b.order, vals, dlo, dhi, coefs);
            void* params[] = {&args};
            cudaKernelNodeParams kp {};
            int const th = group_threads(b, g);
            kp.func = reinterpret_cast<void*>(kernel_of(b.gshape[size_t(g)], b.grefine[size_t(g)] != 0));
            kp.gridDim = dim3(unsigned(group_blocks(b, g, th, b.blocks_per_sm)));
            kp.blockDim = dim3(unsigned(th));
            kp.sharedMemBytes = unsigned(b.gsmem[size_t(g)]);
            kp.kernelParams = params;
            cudaGraphNode_t knode = nullptr;
            DDCB_CUDA_CHECK(cudaGraphAddKernelNode(&knode, b.graph, &mnode, 1, &kp));
            if (b.prio && greatest != least) {
                cudaLaunchAttributeValue v {};
                // numerically lower is higher: the largest group gets `greatest`, the smallest `least`
                v.priority = std::min(least, greatest + b.grank[size_t(g)] * (least - greatest) / std::max(1, b.nrank - 1));
                DDCB_CUDA_CHECK(cudaGraphKernelNodeSetAttribute(knode, cudaLaunchAttributePriority, &v));
            }
            built[size_t(g)] = knode;
        }
        // each group's points are evaluated once its own problems are built, while the other
        // groups may still be building
        for (int g : by_rank) {
            if (b.gnseg[size_t(g)] == 0) continue;
            UnevenEvalArgs ea {b.d_evals, b.d_segs + b.gseg0[size_t(g)], coefs, coords, out};
            void* params[] = {&ea};
            cudaKernelNodeParams kp {};
            kp.func = reinterpret_cast<void*>(uneven_eval_kernel);
            kp.gridDim = dim3(unsigned(b.gnseg[size_t(g)]));
            kp.blockDim = dim3(unsigned(kEvalThreads));
            kp.sharedMemBytes = 0;
            kp.kernelParams = params;
            cudaGraphNode_t enode = nullptr;
            DDCB_CUDA_CHECK(cudaGraphAddKernelNode(&enode, b.graph, &built[size_t(g)], 1, &kp));
        }
        DDCB_CUDA_CHECK(cudaGraphInstantiateWithFlags(&b.exec, b.graph, b.prio ? cudaGraphInstantiateFlagUseNodePriority : 0));
        b.key = key;
        b.key_coords = coords;
        b.key_out = out;
        b.key_stream = s;
        b.key_threads = b.threads;
        b.key_blocks = b.blocks_per_sm;
        b.key_order = b.order;
        b.key_warp = b.warp;
    }
    DDCB_CUDA_CHECK(cudaGraphLaunch(b.exec, s));
}

void tune_uneven_batch(UnevenBatch& b, double const* vals, double const* dlo, double const* dhi, double* coefs,
                       double const* coords, double* out, int reps, cudaStream_t s)
{
    if (b.count == 0) return;
    reps = std::max(1, reps);
    cudaEvent_t e0, e1;
    DDCB_CUDA_CHECK(cudaEventCreate(&e0));
    DDCB_CUDA_CHECK(cudaEventCreate(&e1));
    double best = 1e300;
    int const t0 = b.threads, p0 = b.blocks_per_sm, o0 = b.order, w0 = b.warp;
    int bt = t0, bb = p0, bo = o0, bw = w0;
    try {
        // each candidate runs as the graph it would be launched as (the group kernels concurrent):
        // the warp schedule with per-SM budgets, and the block schedule with block sizes and budgets
        struct Cand
        {
            int warp, threads, per;
        };
        std::vector<Cand> cands;
        for (int per : {0, 1, 2, 4, 8}) cands.push_back({1, 256, per});
        for (int threads : {128, 256, 512})
            for (int per : {1, 2, 4, 8}) cands.push_back({0, threads, per});
        for (Cand const& cd : cands) {
            if (!cd.warp && cd.threads < b.max_chunks) continue; // one thread per chunk of the longest problem
            {
                for (int order : {0, 1}) {
                    b.warp = cd.warp;
                    b.threads = cd.threads;
                    b.blocks_per_sm = cd.per;
                    b.order = order;
                    run_uneven_batch(b, vals, dlo, dhi, coefs, coords, out, s); // builds the graph; warm-up
                    DDCB_CUDA_CHECK(cudaEventRecord(e0, s));
                    for (int r = 0; r < reps; ++r) run_uneven_batch(b, vals, dlo, dhi, coefs, coords, out, s);
                    DDCB_CUDA_CHECK(cudaEventRecord(e1, s));
                    DDCB_CUDA_CHECK(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    DDCB_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                    double const us = 1e3 * ms / reps;
                    if (us < best) {
                        best = us;
                        bt = cd.threads;
                        bb = cd.per;
                        bo = order;
                        bw = cd.warp;
                    }
                }
            }
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b.threads = t0;
        b.blocks_per_sm = p0;
        b.order = o0;
        b.warp = w0;
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b.threads = bt;
    b.blocks_per_sm = bb;
    b.order = bo;
    b.warp = bw;
    if (best < 1e300) b.tuned_us = best;
}

} // namespace ddcb
