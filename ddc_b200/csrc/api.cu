// api.cu -- the extern "C" boundary (include/ddcb.h). Each entry point validates its arguments,
// runs the C++ plan / kernel code and turns every C++ exception into a ddcb_status.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "check_bounds.cuh"
#include "ddcb_internal.hpp"

struct ddcb_bsplines_t
{
    ddcb::Basis basis;
};
struct ddcb_builder_t
{
    ddcb::Builder* b;
    std::mutex quad_mutex;    // guards the first computation of the quadrature weights
    bool quad_ready = false;
};
struct ddcb_evaluator_t
{
    ddcb::Evaluator* e;
};

namespace {

thread_local std::string g_last_error;

// An NVTX range named after the entry point spans each call (the reference labels its regions the
// same way, e.g. spline_builder.hpp:1043), so profilers show the C-ABI calls around their kernels.
struct NvtxRange
{
    explicit NvtxRange(char const* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

template <class F>
ddcb_status guarded(char const* name, F&& f)
{
    NvtxRange const range(name);
    try {
        f();
        g_last_error.clear();
        return DDCB_SUCCESS;
    } catch (ddcb::Error const& e) {
        g_last_error = e.what();
        return e.status;
    } catch (std::bad_alloc const&) {
        g_last_error = "host allocation failed";
        return DDCB_ERR_INVALID_ARGUMENT;
    } catch (std::exception const& e) {
        g_last_error = e.what();
        return DDCB_ERR_INVALID_ARGUMENT;
    }
}

void require(bool ok, char const* what)
{
    if (!ok) throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, what);
}

void check_lines(ddcb_lines const& l, int64_t n_expected, char const* name)
{
    if (l.n != n_expected)
        throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, std::string(name) + ": extent along the interest dimension is "
                                                           + std::to_string(l.n) + ", expected " + std::to_string(n_expected));
    if (l.inner < 0 || l.outer < 0 || l.stride < 0 || l.outer_stride < 0)
        throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, std::string(name) + ": negative extent or stride");
    if (l.inner * l.outer > 0 && l.n > 0 && l.stride == 0)
        throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, std::string(name) + ": zero stride along the interest dimension");
    // 32-bit row index times stride must stay in 64-bit range; batch index fits in the grid
    if (l.inner * l.outer > (int64_t(1) << 40)) throw ddcb::Error(DDCB_ERR_UNSUPPORTED, std::string(name) + ": too many lines");
}

void same_batch(ddcb_lines const& a, ddcb_lines const& b, char const* name)
{
    if (a.inner * a.outer != b.inner * b.outer)
        throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, std::string(name) + ": batch sizes differ");
}

} // namespace

namespace ddcb {

Evaluator* create_evaluator(Basis const& basis, int ex_lo, int ex_hi)
{
    auto* e = new Evaluator();
    try {
        e->basis.desc = basis.desc;
        e->basis.knots = basis.knots;
        e->basis.desc.knots = e->basis.knots.data();
        e->ex_lo = ex_lo;
        e->ex_hi = ex_hi;
        BasisDesc const& D = e->basis.desc;
        int const nk = int(e->basis.knots.size());
        int const d = D.degree;
        auto const& t = e->basis.knots;
        // knot pairs (t_i, t_i+1)
        std::vector<double> kp(size_t(2) * (nk - 1));
        for (int i = 0; i + 1 < nk; ++i) {
            kp[2 * i] = t[i];
            kp[2 * i + 1] = t[i + 1];
        }
        auto inv = [&](long a, long b) { return t[b] > t[a] ? 1.0 / (t[b] - t[a]) : 0.0; };
        // knot-span inverses 1/(t[i+len]-t[i]) for len = 1..d (0 where the span is empty)
        std::vector<double> ispan(size_t(d) * nk, 0.0);
        for (int len = 1; len <= d; ++len)
            for (int i = 0; i + len < nk; ++i) ispan[size_t(len - 1) * nk + i] = inv(i, i + len);
        // bucket table over nb uniform buckets, at least one per cell and, up to 4 per cell and
        // 4096 in all, no wider than the narrowest cell, so that a bucket holds at most one knot:
        // {split, c0} with c0 the cell holding the bucket start and split the first knot inside
        // the bucket (+inf if none)
        int const last = d + D.ncells - 1;
        double hmin = D.rmax - D.rmin;
        for (int cc = d; cc <= last; ++cc) hmin = std::min(hmin, t[cc + 1] - t[cc]);
        double const want = std::ceil((D.rmax - D.rmin) / hmin);
        int const nb = std::max(std::max(1, D.ncells),
                                int(std::min(want, double(std::min(4 * std::max(1, D.ncells), 4096)))));
        std::vector<double> lut(size_t(2) * nb);
        double const scale = double(nb) / (D.rmax - D.rmin);
        int c = d;
        for (int bk = 0; bk < nb; ++bk) {
            double const x0 = D.rmin + double(bk) / scale, x1 = D.rmin + double(bk + 1) / scale;
            while (c < last && x0 >= t[c + 1]) ++c;
            lut[2 * size_t(bk)] = (c < last && t[c + 1] < x1) ? t[c + 1] : HUGE_VAL;
            lut[2 * size_t(bk) + 1] = double(c);
        }
        e->integrals.resize(e->basis.size());
        basis_integrals(e->basis, e->integrals.data());
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        e->device = dev;
        upload_basis(e->basis, dev);
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        size_t const b_kp = kp.size() * 8, b_lut = lut.size() * 8, b_int = e->integrals.size() * 8;
        size_t const b_isp = ispan.size() * 8;
        size_t const o_lut = up(b_kp), o_isp = o_lut + up(b_lut), o_int = o_isp + up(b_isp);
        size_t const total = o_int + b_int + 8;
        DDCB_CUDA_CHECK(cudaMalloc(&e->d_block, total));
        char* base = static_cast<char*>(e->d_block);
        DDCB_CUDA_CHECK(cudaMemcpy(base, kp.data(), b_kp, cudaMemcpyHostToDevice));
        DDCB_CUDA_CHECK(cudaMemcpy(base + o_lut, lut.data(), b_lut, cudaMemcpyHostToDevice));
        DDCB_CUDA_CHECK(cudaMemcpy(base + o_isp, ispan.data(), b_isp, cudaMemcpyHostToDevice));
        DDCB_CUDA_CHECK(cudaMemcpy(base + o_int, e->integrals.data(), b_int, cudaMemcpyHostToDevice));
        e->d_integrals = reinterpret_cast<double*>(base + o_int);
        e->eb.b = e->basis.device_desc();
        e->eb.kpairs = reinterpret_cast<double2 const*>(base);
        e->eb.lut = reinterpret_cast<double2 const*>(base + o_lut);
        e->eb.inv_span = reinterpret_cast<double const*>(base + o_isp);
        e->eb.nbucket = nb;
        e->eb.bucket_scale = scale;
        e->eb.nk = nk;
        return e;
    } catch (...) {
        destroy_evaluator(e);
        throw;
    }
}

void destroy_evaluator(Evaluator* e)
{
    if (!e) return;
    if (e->d_block) cudaFree(e->d_block);
    free_basis(e->basis);
    delete e;
}

// The readers of the translation units' bounds-event words (bounds-checked build only; a
// function-local static, so the units' load-time registrations find it constructed).
std::vector<BoundsReader>& bounds_readers()
{
    static std::vector<BoundsReader> readers;
    return readers;
}

void register_bounds_reader(BoundsReader r) { bounds_readers().push_back(r); }

// The file of a recorded event, from its tag (the device sources and headers that name indices).
std::string bounds_site_name(unsigned long long site)
{
    static char const* const files[] = {"build_device.cuh", "eval_device.cuh", "refine_device.cuh", "adjoint_kernels.cu",
                                        "build_kernels.cu", "eval_kernels.cu", "fused_kernels.cu", "tensor2d.cu",
                                        "tensornd.cu", "uneven_batch.cu", "quadrature.cu", "refine_kernels.cu",
                                        "host_pipeline.cu", "api.cu"};
    uint32_t const tag = uint32_t(site >> 16) & 0xFFFFu;
    std::string name = "unknown file";
    for (char const* f : files)
        if (bounds_file_tag(f) == tag) name = f;
    return name + ":" + std::to_string(site & 0xFFFFull);
}

} // namespace ddcb

extern "C" {

int32_t ddcb_bounds_checked(void)
{
#ifdef DDCB_CHECK_BOUNDS
    return 1;
#else
    return 0;
#endif
}

ddcb_status ddcb_last_device_error(ddcb_stream stream)
{
    return guarded(__func__, [&] {
        cudaError_t const e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
        if (e != cudaSuccess)
            throw ddcb::Error(DDCB_ERR_CUDA, std::string("a kernel queued on this stream failed: ") + cudaGetErrorString(e));
        // every unit's event is read (and so cleared); the first one found is reported
        std::string first;
        for (ddcb::BoundsReader r : ddcb::bounds_readers()) {
            ddcb::BoundsEvent ev {};
            if (r(&ev) && first.empty())
                first = "index " + std::to_string(ev.index) + " outside [0, " + std::to_string(ev.bound) + ") at "
                        + ddcb::bounds_site_name(ev.site) + " (the kernel went on with the index clamped)";
        }
        if (!first.empty()) throw ddcb::Error(DDCB_ERR_DEVICE, first);
    });
}

const char* ddcb_status_string(ddcb_status s)
{
    switch (s) {
    case DDCB_SUCCESS: return "success";
    case DDCB_ERR_INVALID_ARGUMENT: return "invalid argument";
    case DDCB_ERR_BAD_GRID: return "invalid interpolation grid";
    case DDCB_ERR_SINGULAR: return "singular matrix";
    case DDCB_ERR_CUDA: return "CUDA error";
    case DDCB_ERR_UNSUPPORTED: return "unsupported";
    case DDCB_ERR_NOT_CONVERGED: return "not converged";
    case DDCB_ERR_DEVICE: return "device-side failure";
    }
    return "unknown status";
}

const char* ddcb_last_error_message(void) { return g_last_error.c_str(); }

ddcb_status ddcb_bsplines_create_uniform(int32_t degree, int32_t periodic, double rmin, double rmax, int64_t ncells,
                                         ddcb_bsplines* out)
{
    return guarded(__func__, [&] {
        require(out != nullptr, "out is NULL");
        auto* h = new ddcb_bsplines_t();
        try {
            ddcb::make_uniform_basis(h->basis, degree, periodic != 0, rmin, rmax, long(ncells));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

ddcb_status ddcb_bsplines_create_non_uniform(int32_t degree, int32_t periodic, const double* breaks, int64_t nbreaks,
                                             ddcb_bsplines* out)
{
    return guarded(__func__, [&] {
        require(out != nullptr, "out is NULL");
        auto* h = new ddcb_bsplines_t();
        try {
            ddcb::make_non_uniform_basis(h->basis, degree, periodic != 0, breaks, long(nbreaks));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

ddcb_status ddcb_bsplines_destroy(ddcb_bsplines b)
{
    return guarded(__func__, [&] {
        if (!b) return;
        ddcb::free_basis(b->basis);
        delete b;
    });
}

ddcb_status ddcb_bsplines_get_info(ddcb_bsplines b, ddcb_bsplines_info* info)
{
    return guarded(__func__, [&] {
        require(b && info, "NULL argument");
        auto const& d = b->basis.desc;
        info->degree = d.degree;
        info->periodic = d.periodic;
        info->uniform = d.uniform;
        info->ncells = d.ncells;
        info->nbasis = b->basis.nbasis();
        info->size = b->basis.size();
        info->rmin = d.rmin;
        info->rmax = d.rmax;
    });
}

ddcb_status ddcb_bsplines_knots(ddcb_bsplines b, int64_t first, int64_t count, double* out)
{
    return guarded(__func__, [&] {
        require(b && out, "NULL argument");
        require(first >= 0 && count >= 0 && first + count <= int64_t(b->basis.knots.size()), "knot range out of bounds");
        std::copy(b->basis.knots.begin() + first, b->basis.knots.begin() + first + count, out);
    });
}

ddcb_status ddcb_greville_points(ddcb_bsplines b, ddcb_closure lo, ddcb_closure hi, double* points, int64_t capacity,
                                 int64_t* npoints)
{
    return guarded(__func__, [&] {
        require(b && npoints, "NULL argument");
        auto pts = ddcb::greville_points(b->basis, int(lo), int(hi));
        *npoints = int64_t(pts.size());
        if (points) {
            require(capacity >= int64_t(pts.size()), "capacity too small for the interpolation points");
            std::copy(pts.begin(), pts.end(), points);
        }
    });
}

ddcb_status ddcb_bsplines_integrals(ddcb_bsplines b, double* out)
{
    return guarded(__func__, [&] {
        require(b && out, "NULL argument");
        ddcb::basis_integrals(b->basis, out);
    });
}

ddcb_status ddcb_builder_create(ddcb_bsplines basis, const double* interp_points, int64_t npoints, ddcb_closure lo,
                                ddcb_closure hi, const ddcb_builder_options* options, ddcb_builder* out)
{
    return guarded(__func__, [&] {
        require(basis && out, "NULL argument");
        auto* h = new ddcb_builder_t();
        try {
            h->b = ddcb::create_builder(basis->basis, interp_points, long(npoints), int(lo), int(hi), options);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

static void check_device(int device, char const* what);

// The quadrature weights of a builder, computed on its first use (device transposed solve and
// builder adjoint, synchronous), once.
static void ensure_quadrature(ddcb_builder h)
{
    std::lock_guard<std::mutex> lock(h->quad_mutex);
    if (h->quad_ready) return;
    ddcb::compute_device_quadrature(*h->b, h->b->d_quad_scratch, h->b->d_quad);
    h->quad_ready = true;
}

ddcb_status ddcb_builder_device_status(ddcb_builder h, ddcb_stream stream)
{
    ddcb_status st = DDCB_SUCCESS;
    ddcb_status const g = guarded(__func__, [&] {
        require(h != nullptr, "builder is NULL");
        ddcb::Builder const& b = *h->b;
        check_device(b.device, "builder");
        cudaStream_t const s = reinterpret_cast<cudaStream_t>(stream);
        unsigned word = 0;
        DDCB_CUDA_CHECK(cudaMemcpyAsync(&word, b.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        DDCB_CUDA_CHECK(cudaStreamSynchronize(s));
        if (word != 0) {
            DDCB_CUDA_CHECK(cudaMemsetAsync(b.d_status, 0, sizeof(unsigned), s));
            DDCB_CUDA_CHECK(cudaStreamSynchronize(s));
            char msg[160];
            std::snprintf(msg, sizeof msg, "a refined FP32 solve ended with an estimated relative error above %.3g",
                          b.refine_tolerance);
            throw ddcb::Error(DDCB_ERR_NOT_CONVERGED, msg);
        }
    });
    return g != DDCB_SUCCESS ? g : st;
}

ddcb_status ddcb_builder_destroy(ddcb_builder b)
{
    return guarded(__func__, [&] {
        if (!b) return;
        ddcb::destroy_builder(b->b);
        delete b;
    });
}

ddcb_status ddcb_builder_get_info(ddcb_builder h, ddcb_builder_info* info)
{
    return guarded(__func__, [&] {
        require(h && info, "NULL argument");
        ddcb::Builder const& b = *h->b;
        info->nbasis = b.n;
        info->size = b.basis.size();
        info->npoints = int64_t(b.points.size());
        info->nbe_lo = b.nbe_lo;
        info->nbe_hi = b.nbe_hi;
        info->nbv_lo = b.nbv_lo;
        info->nbv_hi = b.nbv_hi;
        info->offset = b.offset;
        info->dx = b.dx;
        info->border = b.k;
        info->kl = b.tables.kl;
        info->ku = b.tables.ku;
        info->pivoting = b.pivot;
        info->chunks = b.tables.nchunk;
        info->tile_lines = b.tile_lines;
    });
}

// Validates a build call; returns false for an empty batch. Clears derivative pointers the
// closures do not read.
static bool check_build(ddcb_builder h, double* coefs, ddcb_lines lc, const double* vals, ddcb_lines lv,
                        const double*& dlo, ddcb_lines llo, const double*& dhi, ddcb_lines lhi)
{
    require(h != nullptr, "builder is NULL");
    ddcb::Builder const& b = *h->b;
    check_lines(lv, int64_t(b.points.size()), "vals");
    check_lines(lc, b.basis.size(), "coefs");
    same_batch(lv, lc, "coefs/vals");
    if (lv.inner * lv.outer == 0) return false; // empty batch: nothing to do (spline_builder.hpp:929-931)
    require(vals && coefs, "vals/coefs pointer is NULL");
    if (b.lo == DDCB_HERMITE && b.nbv_lo > 0) {
        require(dlo != nullptr, "derivs_lo is required by the lower HERMITE closure");
        check_lines(llo, b.nbv_lo, "derivs_lo");
        same_batch(llo, lv, "derivs_lo/vals");
    } else {
        dlo = nullptr;
    }
    if (b.hi == DDCB_HERMITE && b.nbv_hi > 0) {
        require(dhi != nullptr, "derivs_hi is required by the upper HERMITE closure");
        check_lines(lhi, b.nbv_hi, "derivs_hi");
        same_batch(lhi, lv, "derivs_hi/vals");
    } else {
        dhi = nullptr;
    }
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev != b.device) throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, "the builder was created for another device");
    return true;
}

ddcb_status ddcb_build_eval(ddcb_builder h, ddcb_evaluator he, int32_t order, double* coefs, ddcb_lines lc,
                            const double* vals, ddcb_lines lv, const double* dlo, ddcb_lines llo, const double* dhi,
                            ddcb_lines lhi, const double* coords, ddcb_lines lx, double* out, ddcb_lines lo,
                            int32_t* fused, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        if (fused) *fused = 0;
        require(he != nullptr, "evaluator is NULL");
        ddcb::Evaluator const& e = *he->e;
        require(order >= 0 && order <= e.basis.desc.degree, "derivative order must be in 0..degree");
        if (!check_build(h, coefs, lc, vals, lv, dlo, llo, dhi, lhi)) return;
        ddcb::Builder const& b = *h->b;
        require(e.basis.desc.degree == b.basis.desc.degree && e.basis.desc.ncells == b.basis.desc.ncells
                    && e.basis.desc.uniform == b.basis.desc.uniform && e.basis.desc.periodic == b.basis.desc.periodic,
                "builder and evaluator use different bases");
        check_lines(lx, lx.n, "coords");
        check_lines(lo, lx.n, "out");
        same_batch(lx, lo, "coords/out");
        same_batch(lx, lv, "coords/vals");
        if (lx.n == 0) {
            ddcb::launch_build(b, coefs, ddcb::to_lines(lc), vals, ddcb::to_lines(lv), dlo, ddcb::to_lines(llo), dhi,
                               ddcb::to_lines(lhi), reinterpret_cast<cudaStream_t>(stream));
            return;
        }
        require(coords && out, "coords/out pointer is NULL");
        bool const f = ddcb::launch_build_eval(b, e, order, coefs, ddcb::to_lines(lc), vals, ddcb::to_lines(lv), dlo,
                                               ddcb::to_lines(llo), dhi, ddcb::to_lines(lhi), coords, ddcb::to_lines(lx),
                                               out, ddcb::to_lines(lo), reinterpret_cast<cudaStream_t>(stream));
        if (fused) *fused = f ? 1 : 0;
    });
}

ddcb_status ddcb_advect(ddcb_builder h, ddcb_evaluator he, double dt, const double* velocity, int64_t velocity_div,
                        double velocity_const, double* out, ddcb_lines lo, const double* vals, ddcb_lines lv,
                        const double* dlo, ddcb_lines llo, const double* dhi, ddcb_lines lhi, double* coefs, ddcb_lines lc,
                        int32_t* fused, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        if (fused) *fused = 0;
        require(h != nullptr && he != nullptr, "builder or evaluator is NULL");
        ddcb::Builder const& b = *h->b;
        ddcb::Evaluator const& e = *he->e;
        require(e.basis.desc.degree == b.basis.desc.degree && e.basis.desc.ncells == b.basis.desc.ncells
                    && e.basis.desc.uniform == b.basis.desc.uniform && e.basis.desc.periodic == b.basis.desc.periodic,
                "builder and evaluator use different bases");
        require(std::isfinite(dt) && std::isfinite(velocity_const), "dt and velocity_const must be finite");
        // the coefficient output is optional: check it like ddcb_build when given
        double* const c_req = coefs;
        ddcb_lines const lc_req = coefs ? lc : ddcb_lines {b.basis.size(), lv.inner, lv.inner, lv.outer, lv.inner * b.basis.size()};
        double dummy = 0.0;
        if (!check_build(h, coefs ? coefs : &dummy, lc_req, vals, lv, dlo, llo, dhi, lhi)) return;
        check_lines(lo, int64_t(b.points.size()), "out");
        same_batch(lo, lv, "out/vals");
        require(out != nullptr, "out is NULL");
        int64_t const nl = lv.inner * lv.outer;
        if (velocity) require(velocity_div >= 1, "velocity_div must be >= 1");
        ddcb::Lines const lcl = ddcb::to_lines(lc_req);
        bool const f = ddcb::launch_advect(b, e, dt, velocity, velocity_const, velocity ? velocity_div : nl, out,
                                           ddcb::to_lines(lo), vals, ddcb::to_lines(lv), dlo, ddcb::to_lines(llo), dhi,
                                           ddcb::to_lines(lhi), c_req, lcl, reinterpret_cast<cudaStream_t>(stream));
        if (fused) *fused = f ? 1 : 0;
    });
}

ddcb_status ddcb_build(ddcb_builder h, double* coefs, ddcb_lines lc, const double* vals, ddcb_lines lv,
                       const double* dlo, ddcb_lines llo, const double* dhi, ddcb_lines lhi, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        if (!check_build(h, coefs, lc, vals, lv, dlo, llo, dhi, lhi)) return;
        ddcb::Builder const& b = *h->b;
        ddcb::launch_build(b, coefs, ddcb::to_lines(lc), vals, ddcb::to_lines(lv), dlo, ddcb::to_lines(llo), dhi,
                           ddcb::to_lines(lhi), reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_solve_multirhs(ddcb_builder h, double* rhs, int64_t ld, int64_t nrhs, int32_t transpose,
                                ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "builder is NULL");
        require(nrhs >= 0 && ld >= nrhs, "ld must be >= nrhs");
        if (nrhs == 0) return;
        require(rhs != nullptr, "rhs is NULL");
        ddcb::launch_solve_multirhs(*h->b, rhs, long(ld), long(nrhs), transpose != 0, reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_quadrature_coefficients(ddcb_builder h, double* qlo, double* q, double* qhi)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "builder is NULL");
        ddcb::Builder const& b = *h->b;
        require(q != nullptr, "q is NULL");
        require(b.nbv_lo == 0 || qlo != nullptr, "q_derivs_lo is NULL");
        require(b.nbv_hi == 0 || qhi != nullptr, "q_derivs_hi is NULL");
        check_device(b.device, "builder");
        ensure_quadrature(h);
        std::vector<double> all(size_t(b.n));
        DDCB_CUDA_CHECK(cudaMemcpy(all.data(), b.d_quad, sizeof(double) * all.size(), cudaMemcpyDeviceToHost));
        long const nv = b.n - b.nbv_lo - b.nbv_hi;
        std::copy(all.begin(), all.begin() + b.nbv_lo, qlo);
        std::copy(all.begin() + b.nbv_lo, all.begin() + b.nbv_lo + nv, q);
        std::copy(all.begin() + b.nbv_lo + nv, all.end(), qhi);
    });
}

ddcb_status ddcb_quadrature_coefficients_device(ddcb_builder h, double* q_all, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "builder is NULL");
        require(q_all != nullptr, "q_all is NULL");
        ddcb::Builder const& b = *h->b;
        check_device(b.device, "builder");
        ensure_quadrature(h);
        DDCB_CUDA_CHECK(cudaMemcpyAsync(q_all, b.d_quad, sizeof(double) * size_t(b.n), cudaMemcpyDeviceToDevice,
                                        reinterpret_cast<cudaStream_t>(stream)));
    });
}

ddcb_status ddcb_integrate_samples(ddcb_builder h, double* out, int64_t out_outer_stride, const double* vals,
                                   ddcb_lines lv, const double* dlo, ddcb_lines llo, const double* dhi, ddcb_lines lhi,
                                   ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "builder is NULL");
        ddcb::Builder const& b = *h->b;
        check_device(b.device, "builder");
        check_lines(lv, int64_t(b.points.size()), "vals");
        int64_t const nl = lv.inner * lv.outer;
        if (nl == 0) return;
        require(vals != nullptr && out != nullptr, "vals or out is NULL");
        require(lv.outer <= 1 || out_outer_stride >= lv.inner, "out_outer_stride must be >= the inner batch extent");
        bool const her_lo = b.lo == DDCB_HERMITE && b.nbv_lo > 0, her_hi = b.hi == DDCB_HERMITE && b.nbv_hi > 0;
        if (her_lo) {
            require(dlo != nullptr, "derivs_lo is NULL but the lower closure is HERMITE");
            check_lines(llo, b.nbv_lo, "derivs_lo");
            same_batch(lv, llo, "derivs_lo");
        }
        if (her_hi) {
            require(dhi != nullptr, "derivs_hi is NULL but the upper closure is HERMITE");
            check_lines(lhi, b.nbv_hi, "derivs_hi");
            same_batch(lv, lhi, "derivs_hi");
        }
        ensure_quadrature(h);
        ddcb::launch_integrate_samples(b, out, out_outer_stride, vals, ddcb::to_lines(lv), her_lo ? dlo : nullptr,
                                       ddcb::to_lines(llo), her_hi ? dhi : nullptr, ddcb::to_lines(lhi),
                                       reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_evaluator_create(ddcb_bsplines basis, ddcb_extrapolation lo, ddcb_extrapolation hi, ddcb_evaluator* out)
{
    return guarded(__func__, [&] {
        require(basis && out, "NULL argument");
        require(lo >= DDCB_EXTRAP_PERIODIC && lo <= DDCB_EXTRAP_CONSTANT && hi >= DDCB_EXTRAP_PERIODIC && hi <= DDCB_EXTRAP_CONSTANT,
                "unknown extrapolation rule");
        auto* h = new ddcb_evaluator_t();
        try {
            h->e = ddcb::create_evaluator(basis->basis, int(lo), int(hi));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

ddcb_status ddcb_evaluator_destroy(ddcb_evaluator e)
{
    return guarded(__func__, [&] {
        if (!e) return;
        ddcb::destroy_evaluator(e->e);
        delete e;
    });
}

static void eval_common(ddcb_evaluator h, int order, double* out, ddcb_lines lo, const double* coords, ddcb_lines lx,
                        const double* coefs, ddcb_lines lc, ddcb_stream stream)
{
    require(h != nullptr, "evaluator is NULL");
    ddcb::Evaluator const& e = *h->e;
    check_lines(lc, e.basis.size(), "coefs");
    check_lines(lx, lx.n, "coords");
    check_lines(lo, lx.n, "out");
    same_batch(lx, lo, "coords/out");
    same_batch(lx, lc, "coords/coefs");
    if (lx.inner * lx.outer == 0 || lx.n == 0) return;
    require(out && coords && coefs, "NULL data pointer");
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev != e.device) throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, "the evaluator was created for another device");
    ddcb::launch_eval(e, order, out, ddcb::to_lines(lo), coords, ddcb::to_lines(lx), coefs, ddcb::to_lines(lc),
                      reinterpret_cast<cudaStream_t>(stream));
}

ddcb_status ddcb_eval(ddcb_evaluator h, double* out, ddcb_lines lo, const double* coords, ddcb_lines lx,
                      const double* coefs, ddcb_lines lc, ddcb_stream stream)
{
    return guarded(__func__, [&] { eval_common(h, 0, out, lo, coords, lx, coefs, lc, stream); });
}

ddcb_status ddcb_eval_deriv(ddcb_evaluator h, int32_t order, double* out, ddcb_lines lo, const double* coords,
                            ddcb_lines lx, const double* coefs, ddcb_lines lc, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "evaluator is NULL");
        require(order >= 1 && order <= h->e->basis.desc.degree, "derivative order must be in 1..degree");
        eval_common(h, order, out, lo, coords, lx, coefs, lc, stream);
    });
}

ddcb_status ddcb_integrate(ddcb_evaluator h, double* out, int64_t out_outer_stride, const double* coefs, ddcb_lines lc,
                           ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "evaluator is NULL");
        ddcb::Evaluator const& e = *h->e;
        check_lines(lc, e.basis.size(), "coefs");
        if (lc.inner * lc.outer == 0) return;
        require(out && coefs, "NULL data pointer");
        ddcb::launch_integrate(e, out, out_outer_stride, coefs, ddcb::to_lines(lc), reinterpret_cast<cudaStream_t>(stream));
    });
}

// Validates the cotangent outputs of the builder adjoint; clears the derivative pointers the
// closures have no values for.
static void check_build_adjoint_outputs(ddcb::Builder const& b, ddcb_lines lgv, double*& gdlo, ddcb_lines lglo,
                                        double*& gdhi, ddcb_lines lghi)
{
    if (b.lo == DDCB_HERMITE && b.nbv_lo > 0 && gdlo) {
        check_lines(lglo, b.nbv_lo, "g_derivs_lo");
        same_batch(lglo, lgv, "g_derivs_lo/g_vals");
    } else {
        gdlo = nullptr;
    }
    if (b.hi == DDCB_HERMITE && b.nbv_hi > 0 && gdhi) {
        check_lines(lghi, b.nbv_hi, "g_derivs_hi");
        same_batch(lghi, lgv, "g_derivs_hi/g_vals");
    } else {
        gdhi = nullptr;
    }
}

static void check_device(int device, char const* what)
{
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev != device) throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, std::string(what) + " was created for another device");
}

ddcb_status ddcb_build_adjoint(ddcb_builder h, const double* gc, ddcb_lines lgc, double* gv, ddcb_lines lgv,
                               double* gdlo, ddcb_lines lglo, double* gdhi, ddcb_lines lghi, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "builder is NULL");
        ddcb::Builder const& b = *h->b;
        check_lines(lgv, int64_t(b.points.size()), "g_vals");
        check_lines(lgc, b.basis.size(), "g_coefs");
        same_batch(lgv, lgc, "g_coefs/g_vals");
        if (lgv.inner * lgv.outer == 0) return;
        require(gv && gc, "g_vals/g_coefs pointer is NULL");
        check_build_adjoint_outputs(b, lgv, gdlo, lglo, gdhi, lghi);
        check_device(b.device, "the builder");
        ddcb::launch_build_adjoint(b, gc, ddcb::to_lines(lgc), gv, ddcb::to_lines(lgv), gdlo, ddcb::to_lines(lglo), gdhi,
                                   ddcb::to_lines(lghi), reinterpret_cast<cudaStream_t>(stream));
    });
}

// Validates the evaluator-side arguments of an adjoint call (coords, g_out, and coefs / g_coords
// when the coordinate cotangents are wanted).
static void check_eval_adjoint(ddcb::Evaluator const& e, int order, ddcb_lines lx, const double* coefs, ddcb_lines lc,
                               ddcb_lines lgy, const double* gx, ddcb_lines lgx)
{
    require(order == 0 || order == 1, "the adjoint covers order 0 (values) and 1 (first derivatives)");
    require(order <= e.basis.desc.degree, "derivative order must be in 0..degree");
    check_lines(lx, lx.n, "coords");
    check_lines(lgy, lx.n, "g_out");
    same_batch(lx, lgy, "coords/g_out");
    if (gx) {
        require(coefs != nullptr, "coefs is required for g_coords");
        check_lines(lc, e.basis.size(), "coefs");
        check_lines(lgx, lx.n, "g_coords");
        same_batch(lx, lc, "coords/coefs");
        same_batch(lx, lgx, "coords/g_coords");
    }
    check_device(e.device, "the evaluator");
}

ddcb_status ddcb_eval_adjoint(ddcb_evaluator he, int32_t order, const double* coords, ddcb_lines lx, const double* coefs,
                              ddcb_lines lc, const double* gy, ddcb_lines lgy, double* gc, ddcb_lines lgc, double* gx,
                              ddcb_lines lgx, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(he != nullptr, "evaluator is NULL");
        ddcb::Evaluator const& e = *he->e;
        check_lines(lgc, e.basis.size(), "g_coefs");
        same_batch(lx, lgc, "coords/g_coefs");
        if (lx.inner * lx.outer == 0) return;
        check_eval_adjoint(e, order, lx, coefs, lc, lgy, gx, lgx);
        require(gc != nullptr && (coords && gy || lx.n == 0), "NULL data pointer");
        ddcb::launch_eval_adjoint(e, order, coords, ddcb::to_lines(lx), coefs, ddcb::to_lines(lc), gy, ddcb::to_lines(lgy),
                                  gc, ddcb::to_lines(lgc), gx, ddcb::to_lines(lgx), reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_build_eval_adjoint(ddcb_builder h, ddcb_evaluator he, int32_t order, const double* coords,
                                    ddcb_lines lx, const double* coefs, ddcb_lines lc, const double* gy, ddcb_lines lgy,
                                    double* gv, ddcb_lines lgv, double* gdlo, ddcb_lines lglo, double* gdhi,
                                    ddcb_lines lghi, double* gx, ddcb_lines lgx, int32_t* fused, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        if (fused) *fused = 0;
        require(h != nullptr, "builder is NULL");
        require(he != nullptr, "evaluator is NULL");
        ddcb::Builder const& b = *h->b;
        ddcb::Evaluator const& e = *he->e;
        require(e.basis.desc.degree == b.basis.desc.degree && e.basis.desc.ncells == b.basis.desc.ncells
                    && e.basis.desc.uniform == b.basis.desc.uniform && e.basis.desc.periodic == b.basis.desc.periodic,
                "builder and evaluator use different bases");
        check_lines(lgv, int64_t(b.points.size()), "g_vals");
        same_batch(lx, lgv, "coords/g_vals");
        if (lgv.inner * lgv.outer == 0) return;
        require(gv != nullptr && (coords && gy || lx.n == 0), "NULL data pointer");
        check_eval_adjoint(e, order, lx, coefs, lc, lgy, gx, lgx);
        check_build_adjoint_outputs(b, lgv, gdlo, lglo, gdhi, lghi);
        check_device(b.device, "the builder");
        bool const f = ddcb::launch_build_eval_adjoint(
            b, e, order, coords, ddcb::to_lines(lx), coefs, ddcb::to_lines(lc), gy, ddcb::to_lines(lgy), gv,
            ddcb::to_lines(lgv), gdlo, ddcb::to_lines(lglo), gdhi, ddcb::to_lines(lghi), gx, ddcb::to_lines(lgx),
            reinterpret_cast<cudaStream_t>(stream));
        if (fused) *fused = f ? 1 : 0;
    });
}

struct ddcb_uneven_batch_t
{
    ddcb::UnevenBatch* b = nullptr;
};

ddcb_status ddcb_batch_uneven_create(const ddcb_builder* builders, const ddcb_evaluator* evaluators, const int64_t* nevals,
                                     int64_t count, ddcb_uneven_batch* out)
{
    return guarded(__func__, [&] {
        require(out != nullptr, "out is NULL");
        *out = nullptr;
        require(count >= 0 && count < (int64_t(1) << 30), "bad problem count");
        require(count == 0 || (builders && evaluators && nevals), "NULL problem arrays");
        std::vector<ddcb::Builder const*> bl(static_cast<size_t>(count));
        std::vector<ddcb::Evaluator const*> ev(static_cast<size_t>(count));
        for (int64_t i = 0; i < count; ++i) {
            require(builders[i] != nullptr && evaluators[i] != nullptr, "NULL builder or evaluator in the batch");
            bl[size_t(i)] = builders[i]->b;
            ev[size_t(i)] = evaluators[i]->e;
        }
        auto* h = new ddcb_uneven_batch_t();
        try {
            h->b = ddcb::create_uneven_batch(bl.data(), ev.data(), nevals, count);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

ddcb_status ddcb_batch_uneven_destroy(ddcb_uneven_batch h)
{
    return guarded(__func__, [&] {
        if (!h) return;
        ddcb::destroy_uneven_batch(h->b);
        delete h;
    });
}

ddcb_status ddcb_batch_uneven_get_info(ddcb_uneven_batch h, ddcb_uneven_info* info)
{
    return guarded(__func__, [&] {
        require(h != nullptr && info != nullptr, "NULL argument");
        int64_t tot[6];
        int sch[5];
        double us = 0.0;
        ddcb::uneven_info(*h->b, tot, sch, &us);
        info->count = tot[0];
        info->total_vals = tot[1];
        info->total_derivs_lo = tot[2];
        info->total_derivs_hi = tot[3];
        info->total_coefs = tot[4];
        info->total_evals = tot[5];
        info->threads = sch[0];
        info->blocks_per_sm = sch[1];
        info->order = sch[2];
        info->shared_bytes = sch[3];
        info->tuned_us = us;
        info->warp_schedule = sch[4];
    });
}

ddcb_status ddcb_batch_uneven_offsets(ddcb_uneven_batch h, int64_t* vals, int64_t* dlo, int64_t* dhi, int64_t* coefs,
                                      int64_t* evals)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "batch is NULL");
        ddcb::uneven_offsets(*h->b, vals, dlo, dhi, coefs, evals);
    });
}

static void check_uneven_buffers(ddcb_uneven_batch h, const double* vals, const double* dlo, const double* dhi,
                                 double* coefs, const double* coords, double* out)
{
    require(h != nullptr, "batch is NULL");
    int64_t tot[6];
    int sch[5];
    double us;
    ddcb::uneven_info(*h->b, tot, sch, &us);
    require(tot[1] == 0 || vals, "vals is NULL");
    require(tot[2] == 0 || dlo, "derivs_lo is NULL");
    require(tot[3] == 0 || dhi, "derivs_hi is NULL");
    require(tot[4] == 0 || coefs, "coefs is NULL");
    require(tot[5] == 0 || (coords && out), "coords/out is NULL");
}

ddcb_status ddcb_batch_uneven_tune(ddcb_uneven_batch h, const double* vals, const double* dlo, const double* dhi,
                                   double* coefs, const double* coords, double* out, int32_t reps, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        check_uneven_buffers(h, vals, dlo, dhi, coefs, coords, out);
        ddcb::tune_uneven_batch(*h->b, vals, dlo, dhi, coefs, coords, out, reps, reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_batch_uneven_run(ddcb_uneven_batch h, const double* vals, const double* dlo, const double* dhi,
                                  double* coefs, const double* coords, double* out, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        check_uneven_buffers(h, vals, dlo, dhi, coefs, coords, out);
        ddcb::run_uneven_batch(*h->b, vals, dlo, dhi, coefs, coords, out, reinterpret_cast<cudaStream_t>(stream));
    });
}

struct ddcb_host_pipeline_t
{
    ddcb::HostPipeline* p = nullptr;
};

// A host layout the pipeline can cut along the batch: rows of the batch (outer == 1, rows apart by
// at least a row), or one contiguous line per batch index (inner == 1, stride 1).
static void check_host_layout(ddcb_lines const& l, char const* name)
{
    if (l.n == 0 || l.inner * l.outer == 0) return;
    bool const rows = l.outer == 1 && l.stride >= l.inner;
    bool const lines = l.inner == 1 && l.stride == 1 && l.outer_stride >= l.n;
    if (!rows && !lines)
        throw ddcb::Error(DDCB_ERR_UNSUPPORTED, std::string(name)
                                                    + ": host layouts must hold the batch in rows (outer == 1) or one contiguous line "
                                                      "per batch index (inner == 1, stride == 1)");
}

ddcb_status ddcb_host_pipeline_create(ddcb_builder hb, ddcb_evaluator he, int32_t order, int64_t npoints, int64_t slice_lines,
                                      ddcb_host_pipeline* out)
{
    return guarded(__func__, [&] {
        require(hb && he && out, "NULL argument");
        ddcb::Builder const& b = *hb->b;
        ddcb::Evaluator const& e = *he->e;
        require(order >= 0 && order <= e.basis.desc.degree, "derivative order must be in 0..degree");
        require(e.basis.desc.degree == b.basis.desc.degree && e.basis.desc.ncells == b.basis.desc.ncells
                    && e.basis.desc.uniform == b.basis.desc.uniform && e.basis.desc.periodic == b.basis.desc.periodic,
                "builder and evaluator use different bases");
        require(npoints >= 0, "negative number of evaluation points");
        require(slice_lines >= 1 && slice_lines <= (int64_t(1) << 30), "slice_lines must be in 1..2^30");
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        require(dev == b.device && dev == e.device, "the builder and the evaluator must live on the current device");
        auto* h = new ddcb_host_pipeline_t();
        try {
            h->p = ddcb::create_host_pipeline(b, e, int(order), npoints, slice_lines);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

ddcb_status ddcb_host_pipeline_destroy(ddcb_host_pipeline h)
{
    return guarded(__func__, [&] {
        if (!h) return;
        ddcb::destroy_host_pipeline(h->p);
        delete h;
    });
}

ddcb_status ddcb_host_pipeline_run(ddcb_host_pipeline h, const double* vals, ddcb_lines lv, const double* dlo, ddcb_lines llo,
                                   const double* dhi, ddcb_lines lhi, const double* coords, ddcb_lines lx, double* out,
                                   ddcb_lines lo, double* coefs, ddcb_lines lc, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h != nullptr, "pipeline is NULL");
        ddcb::HostPipeline& p = *h->p;
        ddcb::Builder const& b = *p.b;
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        require(dev == p.device, "the pipeline was created for another device");
        check_lines(lv, int64_t(b.points.size()), "vals");
        check_lines(lx, p.m, "coords");
        check_lines(lo, p.m, "out");
        same_batch(lx, lv, "coords/vals");
        same_batch(lo, lv, "out/vals");
        check_host_layout(lv, "vals");
        check_host_layout(lx, "coords");
        check_host_layout(lo, "out");
        if (coefs) {
            check_lines(lc, b.basis.size(), "coefs");
            same_batch(lc, lv, "coefs/vals");
            check_host_layout(lc, "coefs");
        }
        if (b.lo == DDCB_HERMITE && b.nbv_lo > 0) {
            require(dlo != nullptr, "derivs_lo is required by the lower HERMITE closure");
            check_lines(llo, b.nbv_lo, "derivs_lo");
            same_batch(llo, lv, "derivs_lo/vals");
            check_host_layout(llo, "derivs_lo");
        } else {
            dlo = nullptr;
        }
        if (b.hi == DDCB_HERMITE && b.nbv_hi > 0) {
            require(dhi != nullptr, "derivs_hi is required by the upper HERMITE closure");
            check_lines(lhi, b.nbv_hi, "derivs_hi");
            same_batch(lhi, lv, "derivs_hi/vals");
            check_host_layout(lhi, "derivs_hi");
        } else {
            dhi = nullptr;
        }
        int64_t const nbatch = lv.inner * lv.outer;
        if (nbatch == 0) return;
        require(vals != nullptr, "vals pointer is NULL");
        require(p.m == 0 || (coords && out), "coords/out pointer is NULL");
        ddcb::HostArrays a;
        a.vals = vals;
        a.lv = ddcb::to_lines(lv);
        a.dlo = dlo;
        a.llo = ddcb::to_lines(llo);
        a.dhi = dhi;
        a.lhi = ddcb::to_lines(lhi);
        a.coords = coords;
        a.lx = ddcb::to_lines(lx);
        a.out = out;
        a.lo = ddcb::to_lines(lo);
        a.coefs = coefs;
        a.lc = ddcb::to_lines(lc);
        ddcb::run_host_pipeline(p, nbatch, a, reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_build2d_workspace_bytes(ddcb_builder b1, ddcb_builder b2, int64_t nbatch, uint64_t* bytes)
{
    return guarded(__func__, [&] {
        require(b1 && b2 && bytes, "NULL argument");
        require(nbatch >= 0, "negative batch");
        *bytes = nbatch ? ddcb::build2d_workspace_bytes(*b1->b, *b2->b, nbatch) : 0;
    });
}

ddcb_status ddcb_build2d(ddcb_builder h1, ddcb_builder h2, double* coefs, const double* vals, const double* dmin1,
                         const double* dmax1, const double* dmin2, const double* dmax2, const double* m11,
                         const double* m21, const double* m12, const double* m22, int64_t nbatch, void* workspace,
                         uint64_t workspace_bytes, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h1 && h2, "builder is NULL");
        require(nbatch >= 0, "negative batch");
        if (nbatch == 0) return;
        ddcb::Builder const& b1 = *h1->b;
        ddcb::Builder const& b2 = *h2->b;
        require(coefs && vals, "coefs/vals pointer is NULL");
        bool const h1lo = b1.lo == DDCB_HERMITE && b1.nbv_lo > 0, h1hi = b1.hi == DDCB_HERMITE && b1.nbv_hi > 0;
        bool const h2lo = b2.lo == DDCB_HERMITE && b2.nbv_lo > 0, h2hi = b2.hi == DDCB_HERMITE && b2.nbv_hi > 0;
        require(!h1lo || dmin1, "derivs_min1 is required by the lower HERMITE closure of dimension 1");
        require(!h1hi || dmax1, "derivs_max1 is required by the upper HERMITE closure of dimension 1");
        require(!h2lo || dmin2, "derivs_min2 is required by the lower HERMITE closure of dimension 2");
        require(!h2hi || dmax2, "derivs_max2 is required by the upper HERMITE closure of dimension 2");
        require(!(h1lo && h2lo) || m11, "mixed_derivs_min1_min2 is required");
        require(!(h1hi && h2lo) || m21, "mixed_derivs_max1_min2 is required");
        require(!(h1lo && h2hi) || m12, "mixed_derivs_min1_max2 is required");
        require(!(h1hi && h2hi) || m22, "mixed_derivs_max1_max2 is required");
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        require(dev == b1.device && dev == b2.device, "the builders were created for another device");
        size_t const need = ddcb::build2d_workspace_bytes(b1, b2, nbatch);
        cudaStream_t const s = reinterpret_cast<cudaStream_t>(stream);
        void* ws = workspace;
        bool owned = false;
        if (ws == nullptr) {
            DDCB_CUDA_CHECK(cudaMallocAsync(&ws, need, s));
            owned = true;
        } else {
            require(workspace_bytes >= need, "workspace too small (see ddcb_build2d_workspace_bytes)");
        }
        try {
            ddcb::launch_build2d(b1, b2, coefs, vals, h1lo ? dmin1 : nullptr, h1hi ? dmax1 : nullptr, h2lo ? dmin2 : nullptr,
                                 h2hi ? dmax2 : nullptr, (h1lo && h2lo) ? m11 : nullptr, (h1hi && h2lo) ? m21 : nullptr,
                                 (h1lo && h2hi) ? m12 : nullptr, (h1hi && h2hi) ? m22 : nullptr, nbatch,
                                 static_cast<double*>(ws), s, 0, true);
        } catch (...) {
            if (owned) cudaFreeAsync(ws, s);
            throw;
        }
        if (owned) DDCB_CUDA_CHECK(cudaFreeAsync(ws, s));
    });
}

ddcb_status ddcb_eval2d(ddcb_evaluator h1, ddcb_evaluator h2, int32_t o1, int32_t o2, double* out, const double* coords,
                        const double* coefs, int64_t npoints, int64_t nbatch, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h1 && h2, "evaluator is NULL");
        require(npoints >= 0 && nbatch >= 0, "negative size");
        require(o1 >= 0 && o1 <= 1 && o2 >= 0 && o2 <= 1, "2D derivative orders must be 0 or 1");
        if (npoints == 0 || nbatch == 0) return;
        require(out && coords && coefs, "NULL data pointer");
        require((reinterpret_cast<uintptr_t>(coords) & 15) == 0, "coords must be 16-byte aligned (coordinate pairs)");
        ddcb::launch_eval2d(*h1->e, *h2->e, o1, o2, out, coords, coefs, npoints, nbatch, reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_integrate2d(ddcb_evaluator h1, ddcb_evaluator h2, double* out, const double* coefs, int64_t nbatch,
                             ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h1 && h2, "evaluator is NULL");
        require(nbatch >= 0, "negative batch");
        if (nbatch == 0) return;
        require(out && coefs, "NULL data pointer");
        ddcb::launch_integrate2d(*h1->e, *h2->e, out, coefs, nbatch, reinterpret_cast<cudaStream_t>(stream));
    });
}

// No-allocation 2D build (see include/ddcb.h): identical validation to ddcb_build2d, scratch from
// the library's static device array.
ddcb_status ddcb_build2d_static_scratch(ddcb_builder h1, ddcb_builder h2, double* coefs, const double* vals,
                                        const double* dmin1, const double* dmax1, const double* dmin2,
                                        const double* dmax2, const double* m11, const double* m21, const double* m12,
                                        const double* m22, int64_t nbatch, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h1 && h2, "builder is NULL");
        require(nbatch >= 0, "negative batch");
        if (nbatch == 0) return;
        ddcb::Builder const& b1 = *h1->b;
        ddcb::Builder const& b2 = *h2->b;
        require(coefs && vals, "coefs/vals pointer is NULL");
        bool const h1lo = b1.lo == DDCB_HERMITE && b1.nbv_lo > 0, h1hi = b1.hi == DDCB_HERMITE && b1.nbv_hi > 0;
        bool const h2lo = b2.lo == DDCB_HERMITE && b2.nbv_lo > 0, h2hi = b2.hi == DDCB_HERMITE && b2.nbv_hi > 0;
        require(!h1lo || dmin1, "derivs_min1 is required by the lower HERMITE closure of dimension 1");
        require(!h1hi || dmax1, "derivs_max1 is required by the upper HERMITE closure of dimension 1");
        require(!h2lo || dmin2, "derivs_min2 is required by the lower HERMITE closure of dimension 2");
        require(!h2hi || dmax2, "derivs_max2 is required by the upper HERMITE closure of dimension 2");
        require(!(h1lo && h2lo) || m11, "mixed_derivs_min1_min2 is required");
        require(!(h1hi && h2lo) || m21, "mixed_derivs_max1_min2 is required");
        require(!(h1lo && h2hi) || m12, "mixed_derivs_min1_max2 is required");
        require(!(h1hi && h2hi) || m22, "mixed_derivs_max1_max2 is required");
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        require(dev == b1.device && dev == b2.device, "the builders were created for another device");
        ddcb::launch_build2d_static(b1, b2, coefs, vals, h1lo ? dmin1 : nullptr, h1hi ? dmax1 : nullptr,
                                    h2lo ? dmin2 : nullptr, h2hi ? dmax2 : nullptr, (h1lo && h2lo) ? m11 : nullptr,
                                    (h1hi && h2lo) ? m21 : nullptr, (h1lo && h2hi) ? m12 : nullptr,
                                    (h1hi && h2hi) ? m22 : nullptr, nbatch, reinterpret_cast<cudaStream_t>(stream));
    });
}

// ---- 3D builder and N-dimensional evaluator ---------------------------------------------------

// Whether input k1 + 3 k2 + 9 k3 of a 3D build is read: every dimension with a derivative kind
// (1 lower, 2 upper) has a HERMITE closure with derivative inputs on that side.
static bool build3d_reads(ddcb::Builder const* const b[3], int idx)
{
    for (int d = 0; d < 3; ++d, idx /= 3) {
        int const k = idx % 3;
        if (k == 1 && !(b[d]->lo == DDCB_HERMITE && b[d]->nbv_lo > 0)) return false;
        if (k == 2 && !(b[d]->hi == DDCB_HERMITE && b[d]->nbv_hi > 0)) return false;
    }
    return true;
}

ddcb_status ddcb_build3d_workspace_bytes(ddcb_builder b1, ddcb_builder b2, ddcb_builder b3, int64_t nbatch, uint64_t* bytes)
{
    return guarded(__func__, [&] {
        require(b1 && b2 && b3 && bytes, "NULL argument");
        require(nbatch >= 0, "negative batch");
        *bytes = ddcb::build3d_workspace_bytes(*b1->b, *b2->b, *b3->b, nbatch);
    });
}

ddcb_status ddcb_build3d(ddcb_builder h1, ddcb_builder h2, ddcb_builder h3, double* coefs, const double* const* inputs,
                         int64_t nbatch, void* workspace, uint64_t workspace_bytes, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        require(h1 && h2 && h3, "builder is NULL");
        require(nbatch >= 0, "negative batch");
        if (nbatch == 0) return;
        require(coefs && inputs && inputs[0], "coefs / inputs / vals pointer is NULL");
        ddcb::Builder const* const b[3] = {h1->b, h2->b, h3->b};
        const double* in[27];
        for (int i = 0; i < 27; ++i) {
            bool const reads = build3d_reads(b, i);
            in[i] = reads ? inputs[i] : nullptr;
            if (reads && in[i] == nullptr)
                throw ddcb::Error(DDCB_ERR_INVALID_ARGUMENT, "build3d: input " + std::to_string(i)
                                                                 + " (k1 + 3 k2 + 9 k3) is required by the HERMITE closures");
        }
        int dev = 0;
        DDCB_CUDA_CHECK(cudaGetDevice(&dev));
        require(dev == b[0]->device && dev == b[1]->device && dev == b[2]->device, "the builders were created for another device");
        size_t const need = ddcb::build3d_workspace_bytes(*b[0], *b[1], *b[2], nbatch);
        cudaStream_t const s = reinterpret_cast<cudaStream_t>(stream);
        void* ws = workspace;
        bool owned = false;
        if (ws == nullptr) {
            DDCB_CUDA_CHECK(cudaMallocAsync(&ws, need, s));
            owned = true;
        } else {
            require(workspace_bytes >= need, "workspace too small (see ddcb_build3d_workspace_bytes)");
        }
        try {
            ddcb::launch_build3d(*b[0], *b[1], *b[2], coefs, in, nbatch, static_cast<double*>(ws), s);
        } catch (...) {
            if (owned) cudaFreeAsync(ws, s);
            throw;
        }
        if (owned) DDCB_CUDA_CHECK(cudaFreeAsync(ws, s));
    });
}

static void evaluators_nd(const ddcb_evaluator* evaluators, int32_t ndims, ddcb::Evaluator const** e)
{
    require(evaluators != nullptr, "evaluators is NULL");
    require(ndims >= 1 && ndims <= ddcb::kMaxDims, "ndims must be in 1..6");
    int dev = 0;
    DDCB_CUDA_CHECK(cudaGetDevice(&dev));
    for (int d = 0; d < ndims; ++d) {
        require(evaluators[d] != nullptr, "evaluator is NULL");
        e[d] = evaluators[d]->e;
        require(e[d]->device == dev, "an evaluator was created for another device");
    }
}

ddcb_status ddcb_evalnd(const ddcb_evaluator* evaluators, int32_t ndims, const int32_t* orders, double* out,
                        const double* coords, const double* coefs, int64_t npoints, int64_t nbatch, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        ddcb::Evaluator const* e[ddcb::kMaxDims] = {};
        evaluators_nd(evaluators, ndims, e);
        require(npoints >= 0 && nbatch >= 0, "negative size");
        int ord[ddcb::kMaxDims] = {};
        if (orders)
            for (int d = 0; d < ndims; ++d) {
                require(orders[d] >= 0 && orders[d] <= e[d]->basis.desc.degree, "derivative order outside 0..degree");
                ord[d] = orders[d];
            }
        if (npoints == 0 || nbatch == 0) return;
        require(out && coords && coefs, "NULL data pointer");
        ddcb::launch_evalnd(e, ndims, orders ? ord : nullptr, out, coords, coefs, npoints, nbatch,
                            reinterpret_cast<cudaStream_t>(stream));
    });
}

ddcb_status ddcb_integratend(const ddcb_evaluator* evaluators, int32_t ndims, double* out, const double* coefs,
                             int64_t nbatch, ddcb_stream stream)
{
    return guarded(__func__, [&] {
        ddcb::Evaluator const* e[ddcb::kMaxDims] = {};
        evaluators_nd(evaluators, ndims, e);
        require(nbatch >= 0, "negative batch");
        if (nbatch == 0) return;
        require(out && coefs, "NULL data pointer");
        ddcb::launch_integratend(e, ndims, out, coefs, nbatch, reinterpret_cast<cudaStream_t>(stream));
    });
}

} // extern "C"
