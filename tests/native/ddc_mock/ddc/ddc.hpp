// A minimal stand-in for the part of DDC's public surface (CExA-project/ddc, src/ddc/) that the
// B200 adapter header uses: discrete elements / vectors / domains, ChunkSpan with its allocation
// mdspan, discrete spaces with coordinates, and the domain type helpers. Test infrastructure only:
// it lets tests compile and run include/ddc_b200/spline_builder_b200.hpp without Kokkos. Names and
// meanings follow DDC (discrete_domain.hpp, chunk_span.hpp, discrete_space.hpp); the storage is
// plain host/device pointers.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <type_traits>
#include <vector>

namespace Kokkos {
struct layout_right {};
struct DefaultExecutionSpace
{
    using memory_space = struct CudaSpaceMock {};
};
} // namespace Kokkos

namespace ddc {

namespace detail {
template <class... T>
struct TypeSeq
{
};
template <class Q, class Seq>
struct Rank;
template <class Q>
struct Rank<Q, TypeSeq<>>
{
    static constexpr std::size_t value = std::numeric_limits<std::size_t>::max();
};
template <class Q, class H, class... T>
struct Rank<Q, TypeSeq<H, T...>>
{
    static constexpr std::size_t rest = Rank<Q, TypeSeq<T...>>::value;
    static constexpr std::size_t value
            = std::is_same_v<Q, H> ? 0 : (rest == std::numeric_limits<std::size_t>::max() ? rest : 1 + rest);
};
} // namespace detail

template <class Q, class Seq>
constexpr std::size_t type_seq_rank_v = detail::Rank<Q, Seq>::value;

template <class CDim>
struct Deriv
{
};

// Coordinate<X>: one double tagged by its continuous dimension.
template <class... CDims>
struct Coordinate
{
    std::array<double, sizeof...(CDims)> v {};
    Coordinate() = default;
    explicit Coordinate(double x) requires(sizeof...(CDims) == 1) : v {x} {}
    operator double() const requires(sizeof...(CDims) == 1) { return v[0]; }
};

template <class DDim>
struct DiscreteVector
{
    std::ptrdiff_t n = 0;
    explicit DiscreteVector(std::ptrdiff_t v = 0) : n(v) {}
    std::ptrdiff_t value() const { return n; }
};

template <class... DDims>
struct DiscreteElement
{
    std::array<std::ptrdiff_t, sizeof...(DDims)> idx {};
    DiscreteElement() = default;
    explicit DiscreteElement(std::ptrdiff_t i) requires(sizeof...(DDims) == 1) : idx {i} {}
    std::ptrdiff_t uid() const requires(sizeof...(DDims) == 1) { return idx[0]; }
};

template <class... DDims>
class DiscreteDomain
{
public:
    static constexpr std::size_t rank() { return sizeof...(DDims); }
    std::array<std::ptrdiff_t, sizeof...(DDims)> front_ {};
    std::array<std::ptrdiff_t, sizeof...(DDims)> ext_ {};

    DiscreteDomain() = default;
    // product of 1D domains, or the restriction of a larger domain to these dimensions
    template <class... Doms>
    explicit DiscreteDomain(Doms const&... doms) requires(sizeof...(Doms) >= 1)
    {
        (take(doms), ...);
    }
    DiscreteDomain(DiscreteElement<DDims...> const& f, DiscreteVector<DDims> const&... n) requires(sizeof...(DDims) == 1)
    {
        front_ = f.idx;
        ext_ = {n.value()...};
    }
    std::size_t size() const
    {
        std::size_t s = 1;
        for (auto e : ext_) s *= std::size_t(e);
        return s;
    }
    template <class DDim>
    std::ptrdiff_t extent() const { return ext_[type_seq_rank_v<DDim, detail::TypeSeq<DDims...>>]; }
    template <class DDim>
    std::ptrdiff_t front_of() const { return front_[type_seq_rank_v<DDim, detail::TypeSeq<DDims...>>]; }
    DiscreteElement<DDims...> front() const
    {
        DiscreteElement<DDims...> e;
        e.idx = front_;
        return e;
    }
    bool operator==(DiscreteDomain const& o) const { return front_ == o.front_ && ext_ == o.ext_; }

    // iteration over a 1D domain
    struct iterator
    {
        std::ptrdiff_t i;
        DiscreteElement<DDims...> operator*() const requires(sizeof...(DDims) == 1) { return DiscreteElement<DDims...>(i); }
        iterator& operator++() { ++i; return *this; }
        bool operator!=(iterator const& o) const { return i != o.i; }
    };
    iterator begin() const requires(sizeof...(DDims) == 1) { return {front_[0]}; }
    iterator end() const requires(sizeof...(DDims) == 1) { return {front_[0] + ext_[0]}; }

private:
    template <class... Others>
    void take(DiscreteDomain<Others...> const& d)
    {
        std::size_t k = 0;
        ((copy_if<Others>(d.front_[k], d.ext_[k]), ++k), ...);
    }
    template <class D>
    void copy_if(std::ptrdiff_t f, std::ptrdiff_t e)
    {
        constexpr std::size_t r = type_seq_rank_v<D, detail::TypeSeq<DDims...>>;
        if constexpr (r < sizeof...(DDims)) {
            front_[r] = f;
            ext_[r] = e;
        }
    }
};

template <class T>
struct ToTypeSeq;
template <class... D>
struct ToTypeSeq<DiscreteDomain<D...>>
{
    using type = detail::TypeSeq<D...>;
};
template <class T>
using to_type_seq_t = typename ToTypeSeq<T>::type;

namespace detail {
template <class Old, class New, class D>
using Swap = std::conditional_t<std::is_same_v<D, Old>, New, D>;
template <class Dom, class Old, class New>
struct Replace;
template <class... D, class Old, class New>
struct Replace<DiscreteDomain<D...>, Old, New>
{
    using type = DiscreteDomain<Swap<Old, New, D>...>;
};
template <class Acc, class Rest, class Rm>
struct Remove;
template <class... A, class Rm>
struct Remove<TypeSeq<A...>, TypeSeq<>, Rm>
{
    using type = DiscreteDomain<A...>;
};
template <class... A, class H, class... T, class... Rm>
struct Remove<TypeSeq<A...>, TypeSeq<H, T...>, TypeSeq<Rm...>>
{
    using type = typename Remove<std::conditional_t<(std::is_same_v<H, Rm> || ...), TypeSeq<A...>, TypeSeq<A..., H>>,
                                 TypeSeq<T...>, TypeSeq<Rm...>>::type;
};
} // namespace detail

template <class Dom, class Old, class New>
using replace_dim_of_t = typename detail::Replace<Dom, Old, New>::type;
template <class Dom, class... Rm>
using remove_dims_of_t = typename detail::Remove<detail::TypeSeq<>, to_type_seq_t<Dom>, detail::TypeSeq<Rm...>>::type;

// Replace in dom_a the dimension Old by the dimension New of dom_b (discrete_domain.hpp:527-552).
template <class Old, class New, class... DA, class... DB>
auto replace_dim_of(DiscreteDomain<DA...> const& a, DiscreteDomain<DB...> const& b)
{
    replace_dim_of_t<DiscreteDomain<DA...>, Old, New> r;
    constexpr std::size_t k = type_seq_rank_v<Old, detail::TypeSeq<DA...>>;
    r.front_ = a.front_;
    r.ext_ = a.ext_;
    r.front_[k] = b.template front_of<New>();
    r.ext_[k] = b.template extent<New>();
    return r;
}
template <class... Rm, class... DA>
auto remove_dims_of(DiscreteDomain<DA...> const& a)
{
    return remove_dims_of_t<DiscreteDomain<DA...>, Rm...>(a);
}

// discrete_space<DDim>(): the mock keeps one instance per dimension type (DDim::Impl).
template <class DDim>
typename DDim::Impl& discrete_space()
{
    static typename DDim::Impl impl;
    return impl;
}
template <class DDim>
Coordinate<typename DDim::continuous_dimension_type> coordinate(DiscreteElement<DDim> const& e)
{
    return Coordinate<typename DDim::continuous_dimension_type>(discrete_space<DDim>().coordinate(e.uid()));
}

// ChunkSpan over a contiguous or strided allocation; allocation_mdspan() exposes extents / strides.
template <std::size_t R>
struct MdspanMock
{
    std::array<std::ptrdiff_t, R> ext {}, str {};
    std::size_t extent(std::size_t r) const { return std::size_t(ext[r]); }
    std::size_t stride(std::size_t r) const { return std::size_t(str[r]); }
};

template <class T, class Dom, class Layout = Kokkos::layout_right, class Mem = Kokkos::DefaultExecutionSpace::memory_space>
class ChunkSpan
{
public:
    T* ptr = nullptr;
    Dom dom {};
    MdspanMock<Dom::rank()> md {};
    ChunkSpan() = default;
    // row-major (layout_right) view of ptr over dom
    ChunkSpan(T* p, Dom const& d) : ptr(p), dom(d)
    {
        std::ptrdiff_t s = 1;
        for (std::size_t r = Dom::rank(); r-- > 0;) {
            md.ext[r] = d.ext_[r];
            md.str[r] = s;
            s *= d.ext_[r];
        }
    }
    ChunkSpan(T* p, Dom const& d, std::array<std::ptrdiff_t, Dom::rank()> const& strides) : ChunkSpan(p, d) { md.str = strides; }
    template <class U>
    ChunkSpan(ChunkSpan<U, Dom, Layout, Mem> const& o) requires std::is_same_v<std::remove_const_t<T>, U>
        : ptr(o.ptr), dom(o.dom), md(o.md)
    {
    }
    Dom domain() const { return dom; }
    T* data_handle() const { return ptr; }
    MdspanMock<Dom::rank()> allocation_mdspan() const { return md; }
    ChunkSpan<T const, Dom, Layout, Mem> span_cview() const { return ChunkSpan<T const, Dom, Layout, Mem>(*this); }
};

} // namespace ddc
