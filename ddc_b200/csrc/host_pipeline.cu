// host_pipeline.cu -- the build + evaluate step on HOST buffers, with the host<->device copies of
// neighbouring batch slices overlapping the kernels.
//
// A DDC user with host data copies it to the device (ddc::parallel_deepcopy), calls
// SplineBuilder::operator() and SplineEvaluator::deriv (examples/characteristics_advection.cpp:
// 251-259) and copies the result back, one step after the other. Here the batch is cut into
// slices of lines; slice i is copied in on one stream, built and evaluated on a second and copied
// out on a third, so the two copy engines and the kernels of slices i-1, i and i+1 run at once and
// the step takes about as long as its larger copy direction. Two device buffer sets alternate
// between slices; events order the reuse of a set after the kernels and the copy-out of the slice
// that used it last (the previous run's slices for a run's first two). Everything is allocated at
// creation: a run allocates nothing.
#include <algorithm>

#include "ddcb_internal.hpp"

namespace ddcb {

namespace {

// One array's host layout cut along the batch: lines [b0, b0 + nb) copied to or from a device
// buffer that keeps the same kind of layout with nb lines.
Lines slice_layout(Lines const& host, int64_t nb)
{
    if (host.outer == 1) return Lines {host.n, nb, nb, 1, 0}; // (x, batch): n rows of nb values
    return Lines {host.n, 1, 1, nb, host.n};                  // (batch, x): nb lines of n values
}

// Copies lines [b0, b0 + nb) of a host array (layout hl) to or from the device buffer dev (layout
// dl = slice_layout(hl, nb)).
void copy_slice(double* dev, Lines const& dl, const double* host, Lines const& hl, int64_t b0, int64_t nb, bool to_device,
                cudaStream_t s)
{
    if (hl.n == 0 || nb == 0) return;
    double* const h = const_cast<double*>(host);
    size_t hpitch, dpitch, width, height;
    double* hb;
    if (hl.outer == 1) { // rows of nb contiguous doubles
        hb = h + b0;
        hpitch = size_t(hl.stride) * 8;
        dpitch = size_t(nb) * 8;
        width = size_t(nb) * 8;
        height = size_t(hl.n);
    } else { // nb lines of n contiguous doubles
        hb = h + b0 * hl.outer_stride;
        hpitch = size_t(hl.outer_stride) * 8;
        dpitch = size_t(dl.n) * 8;
        width = size_t(hl.n) * 8;
        height = size_t(nb);
    }
    if (to_device) DDCB_CUDA_CHECK(cudaMemcpy2DAsync(dev, dpitch, hb, hpitch, width, height, cudaMemcpyHostToDevice, s));
    else DDCB_CUDA_CHECK(cudaMemcpy2DAsync(hb, hpitch, dev, dpitch, width, height, cudaMemcpyDeviceToHost, s));
}

} // namespace

HostPipeline* create_host_pipeline(Builder const& b, Evaluator const& e, int order, int64_t m, int64_t slice)
{
    auto* p = new HostPipeline();
    try {
        p->b = &b;
        p->e = &e;
        p->order = order;
        p->m = m;
        p->slice = slice;
        DDCB_CUDA_CHECK(cudaGetDevice(&p->device));
        int64_t const np = int64_t(b.points.size()), size = b.basis.size();
        // per buffer set, in doubles: vals, derivs_lo, derivs_hi, coords, out, coefs
        int64_t const rows[6] = {np, b.nbv_lo, b.nbv_hi, m, m, size};
        size_t off = 0;
        size_t offs[2][6];
        for (int k = 0; k < 2; ++k)
            for (int a = 0; a < 6; ++a) {
                offs[k][a] = off;
                off += (size_t(rows[a]) * size_t(slice) * 8 + 255) / 256 * 256;
            }
        DDCB_CUDA_CHECK(cudaMalloc(&p->d_block, std::max<size_t>(off, 256)));
        char* base = static_cast<char*>(p->d_block);
        for (int k = 0; k < 2; ++k)
            for (int a = 0; a < 6; ++a) p->buf[k][a] = reinterpret_cast<double*>(base + offs[k][a]);
        DDCB_CUDA_CHECK(cudaStreamCreateWithFlags(&p->s_in, cudaStreamNonBlocking));
        DDCB_CUDA_CHECK(cudaStreamCreateWithFlags(&p->s_comp, cudaStreamNonBlocking));
        DDCB_CUDA_CHECK(cudaStreamCreateWithFlags(&p->s_out, cudaStreamNonBlocking));
        DDCB_CUDA_CHECK(cudaEventCreateWithFlags(&p->ev_start, cudaEventDisableTiming));
        for (int k = 0; k < 2; ++k) {
            DDCB_CUDA_CHECK(cudaEventCreateWithFlags(&p->in_done[k], cudaEventDisableTiming));
            DDCB_CUDA_CHECK(cudaEventCreateWithFlags(&p->comp_done[k], cudaEventDisableTiming));
            DDCB_CUDA_CHECK(cudaEventCreateWithFlags(&p->out_done[k], cudaEventDisableTiming));
        }
        return p;
    } catch (...) {
        destroy_host_pipeline(p);
        throw;
    }
}

void destroy_host_pipeline(HostPipeline* p)
{
    if (!p) return;
    // the streams may still run a pipeline's last slices
    if (p->s_out) cudaStreamSynchronize(p->s_out);
    if (p->s_comp) cudaStreamSynchronize(p->s_comp);
    if (p->s_in) cudaStreamSynchronize(p->s_in);
    for (int k = 0; k < 2; ++k) {
        if (p->in_done[k]) cudaEventDestroy(p->in_done[k]);
        if (p->comp_done[k]) cudaEventDestroy(p->comp_done[k]);
        if (p->out_done[k]) cudaEventDestroy(p->out_done[k]);
    }
    if (p->ev_start) cudaEventDestroy(p->ev_start);
    if (p->s_in) cudaStreamDestroy(p->s_in);
    if (p->s_comp) cudaStreamDestroy(p->s_comp);
    if (p->s_out) cudaStreamDestroy(p->s_out);
    if (p->d_block) cudaFree(p->d_block);
    delete p;
}

void run_host_pipeline(HostPipeline& p, int64_t nbatch, HostArrays const& h, cudaStream_t user)
{
    Builder const& b = *p.b;
    Evaluator const& e = *p.e;
    // the pipeline's streams start after the work already queued on the caller's stream
    DDCB_CUDA_CHECK(cudaEventRecord(p.ev_start, user));
    DDCB_CUDA_CHECK(cudaStreamWaitEvent(p.s_in, p.ev_start, 0));
    DDCB_CUDA_CHECK(cudaStreamWaitEvent(p.s_out, p.ev_start, 0));
    int64_t const nslices = (nbatch + p.slice - 1) / p.slice;
    for (int64_t i = 0; i < nslices; ++i) {
        int const k = int(i % 2);
        int64_t const b0 = i * p.slice, nb = std::min(p.slice, nbatch - b0);
        double* const* d = p.buf[k];
        Lines const lv = slice_layout(h.lv, nb), llo = slice_layout(h.llo, nb), lhi = slice_layout(h.lhi, nb);
        Lines const lx = slice_layout(h.lx, nb), lo = slice_layout(h.lo, nb);
        Lines const lc = h.coefs ? slice_layout(h.lc, nb) : Lines {b.basis.size(), nb, nb, 1, 0};
        // copy in once the kernels of the slice that last used this buffer set have read it (an
        // event never recorded is complete)
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(p.s_in, p.comp_done[k], 0));
        copy_slice(d[0], lv, h.vals, h.lv, b0, nb, true, p.s_in);
        if (h.dlo) copy_slice(d[1], llo, h.dlo, h.llo, b0, nb, true, p.s_in);
        if (h.dhi) copy_slice(d[2], lhi, h.dhi, h.lhi, b0, nb, true, p.s_in);
        copy_slice(d[3], lx, h.coords, h.lx, b0, nb, true, p.s_in);
        DDCB_CUDA_CHECK(cudaEventRecord(p.in_done[k], p.s_in));
        // build and evaluate once the inputs are in and the outputs of that slice are out
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(p.s_comp, p.in_done[k], 0));
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(p.s_comp, p.out_done[k], 0));
        if (lx.n > 0)
            launch_build_eval(b, e, p.order, d[5], lc, d[0], lv, h.dlo ? d[1] : nullptr, llo, h.dhi ? d[2] : nullptr, lhi, d[3], lx,
                              d[4], lo, p.s_comp);
        else
            launch_build(b, d[5], lc, d[0], lv, h.dlo ? d[1] : nullptr, llo, h.dhi ? d[2] : nullptr, lhi, p.s_comp);
        DDCB_CUDA_CHECK(cudaEventRecord(p.comp_done[k], p.s_comp));
        // copy out
        DDCB_CUDA_CHECK(cudaStreamWaitEvent(p.s_out, p.comp_done[k], 0));
        copy_slice(d[4], lo, h.out, h.lo, b0, nb, false, p.s_out);
        if (h.coefs) copy_slice(d[5], lc, h.coefs, h.lc, b0, nb, false, p.s_out);
        DDCB_CUDA_CHECK(cudaEventRecord(p.out_done[k], p.s_out));
    }
    // the caller's stream continues once the last slice is out (the copy-out stream is in order,
    // and its last copy followed the last kernels)
    if (nslices > 0) DDCB_CUDA_CHECK(cudaStreamWaitEvent(user, p.out_done[(nslices - 1) % 2], 0));
}

} // namespace ddcb
