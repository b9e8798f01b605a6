// check_bounds.cuh -- the index checks of the DDCB_CHECK_BOUNDS build.
//
// The reference's debug builds assert the ranges of the basis indices they compute
// (KOKKOS_ASSERT, bsplines_uniform.hpp:489-494, bsplines_non_uniform.hpp:469-479). Here the
// kernels name each computed index they use to address an array -- a cell, a knot pair, a tile
// row, a problem -- through DDCB_INDEX(i, n). In a library built with -DDDCB_CHECK_BOUNDS
// (libddcb_check.so), an index outside [0, n) is recorded in a device word of the translation
// unit (the first event per query wins: the site's file and line, the index and the bound) and the
// kernel goes on with the index clamped into range: no trap, no device assert, no access outside
// the array. ddcb_last_device_error reads and clears the words of every translation unit. In the
// default build DDCB_INDEX is the index itself.
#pragma once

#include <cstdint>

namespace ddcb {

// 16-bit hash of a file's base name (FNV-1a): the site tag of a recorded event.
constexpr uint32_t bounds_file_tag(const char* path)
{
    const char* base = path;
    for (const char* p = path; *p; ++p)
        if (*p == '/') base = p + 1;
    uint32_t h = 2166136261u;
    for (const char* p = base; *p; ++p) h = (h ^ uint32_t(static_cast<unsigned char>(*p))) * 16777619u;
    return (h ^ (h >> 16)) & 0xFFFFu;
}

// One recorded event: site = file tag << 16 | line (0: none).
struct BoundsEvent
{
    unsigned long long site;
    long long index;
    long long bound;
};

// Reads and clears one translation unit's event on the current device (registered at load time).
using BoundsReader = bool (*)(BoundsEvent*);
void register_bounds_reader(BoundsReader r);

} // namespace ddcb

#if defined(DDCB_CHECK_BOUNDS) && defined(__CUDACC__)

#include <cuda_runtime.h>

namespace ddcb {
namespace {

__device__ unsigned long long g_bounds_site;
__device__ long long g_bounds_index;
__device__ long long g_bounds_bound;

__device__ __forceinline__ long long bounds_checked(long long i, long long n, unsigned long long site)
{
    if (i >= 0 && i < n) return i;
    if (atomicCAS(&g_bounds_site, 0ull, site) == 0ull) {
        g_bounds_index = i;
        g_bounds_bound = n;
    }
    return i < 0 || n <= 0 ? 0 : n - 1;
}

bool read_bounds_event(BoundsEvent* e)
{
    unsigned long long site = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&site, g_bounds_site, sizeof(site)) != cudaSuccess || site == 0) return false;
    cudaMemcpyFromSymbol(&e->index, g_bounds_index, sizeof(e->index));
    cudaMemcpyFromSymbol(&e->bound, g_bounds_bound, sizeof(e->bound));
    e->site = site;
    cudaMemcpyToSymbol(g_bounds_site, &zero, sizeof(zero));
    return true;
}

struct BoundsRegistration
{
    BoundsRegistration() { register_bounds_reader(&read_bounds_event); }
};
BoundsRegistration const g_bounds_registration;

} // namespace
} // namespace ddcb

#define DDCB_INDEX(i, n)                                                                                         \
    static_cast<decltype(i)>(::ddcb::bounds_checked(static_cast<long long>(i), static_cast<long long>(n),       \
                                                    (static_cast<unsigned long long>(::ddcb::bounds_file_tag(__FILE__)) << 16) | \
                                                        static_cast<unsigned long long>(__LINE__)))

#else

#define DDCB_INDEX(i, n) (i)

#endif
