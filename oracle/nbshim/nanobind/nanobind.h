// Minimal nanobind-compatible shim used ONLY to compile the reference's own
// native sources (gwldcore.cpp, winldcore.cpp) unchanged into a plain C++
// shared library for parity checks and the CPU baseline.  It is test
// infrastructure: nothing in the product links it.
//
// Only the API surface those two translation units use is provided:
// ndarray views over caller-owned memory, a type-erased `object` that is
// either None, an integer, a float, a string or an array, `cast`, `dict`,
// `tuple`/`make_tuple`, `capsule`, GIL guards (no-ops), `python_error`, and
// an NB_MODULE that registers nothing.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

// The reference polls Ctrl-C through the CPython API; the harness never has
// a pending signal.
inline int PyErr_CheckSignals() { return 0; }

namespace nanobind {

struct dlpack_dtype {
    uint8_t code = 0;   // 0 int, 1 uint, 2 float
    uint8_t bits = 0;
    uint16_t lanes = 1;
    bool operator==(const dlpack_dtype& o) const {
        return code == o.code && bits == o.bits && lanes == o.lanes;
    }
    bool operator!=(const dlpack_dtype& o) const { return !(*this == o); }
};

template <typename T>
inline dlpack_dtype dtype() {
    using U = std::remove_cv_t<T>;
    dlpack_dtype d;
    d.bits = (uint8_t)(sizeof(U) * 8);
    if constexpr (std::is_floating_point_v<U>) d.code = 2;
    else if constexpr (std::is_signed_v<U>) d.code = 0;
    else d.code = 1;
    return d;
}

namespace device { struct cpu {}; }
struct c_contig {};
struct f_contig {};
struct numpy {};
struct ro {};
template <size_t N> struct ndim {};
template <ptrdiff_t... S> struct shape {};

class capsule {
public:
    capsule() = default;
    capsule(void* p, void (*del)(void*) noexcept) : owner_(p, del) {}
    std::shared_ptr<void> owner_;
};

// Type-erased array description shared by ndarray<> and object.
struct array_desc {
    void* data = nullptr;
    size_t ndim = 0;
    size_t shape[4] = {0, 0, 0, 0};
    dlpack_dtype dt;
    std::shared_ptr<void> owner;
};

namespace detail {
template <typename... Ts> struct first_scalar { using type = void; };
template <typename T, typename... Ts> struct first_scalar<T, Ts...> {
    using U = std::remove_cv_t<T>;
    using type = std::conditional_t<std::is_arithmetic_v<U>, T,
                                    typename first_scalar<Ts...>::type>;
};
}  // namespace detail

template <typename Scalar>
struct ndarray_view1 {
    Scalar* p = nullptr;
    Scalar& operator()(size_t i) const { return p[i]; }
};

template <typename... Args>
class ndarray {
public:
    using Scalar = typename detail::first_scalar<Args...>::type;
    array_desc d;

    ndarray() = default;
    explicit ndarray(const array_desc& desc) : d(desc) {}
    template <typename P>
    ndarray(P* ptr, std::initializer_list<size_t> shp, capsule owner = capsule()) {
        d.data = (void*)ptr;
        d.ndim = shp.size();
        size_t i = 0;
        for (size_t s : shp) d.shape[i++] = s;
        d.dt = ::nanobind::dtype<std::remove_cv_t<P>>();
        d.owner = owner.owner_;
    }

    Scalar* data() const { return static_cast<Scalar*>(d.data); }
    size_t shape(size_t i) const { return d.shape[i]; }
    size_t ndim() const { return d.ndim; }
    dlpack_dtype dtype() const { return d.dt; }
    size_t size() const {
        size_t n = 1;
        for (size_t i = 0; i < d.ndim; ++i) n *= d.shape[i];
        return n;
    }
    template <typename U, typename... Rest>
    ndarray_view1<U> view() const { return ndarray_view1<U>{static_cast<U*>(d.data)}; }
};

class object {
public:
    enum class Kind { None, Int, Float, Str, Array };
    object() = default;
    static object from_int(int64_t v) { object o; o.kind_ = Kind::Int; o.i_ = v; return o; }
    static object from_uint(uint64_t v) { object o; o.kind_ = Kind::Int; o.u_ = v; o.i_ = (int64_t)v; return o; }
    static object from_float(double v) { object o; o.kind_ = Kind::Float; o.f_ = v; return o; }
    static object from_array(const array_desc& a) { object o; o.kind_ = Kind::Array; o.a_ = a; return o; }
    template <typename... A>
    object(const ndarray<A...>& arr) : kind_(Kind::Array), a_(arr.d) {}

    bool is_none() const { return kind_ == Kind::None; }
    Kind kind() const { return kind_; }
    int64_t i_ = 0;
    uint64_t u_ = 0;
    double f_ = 0.0;
    array_desc a_;
private:
    Kind kind_ = Kind::None;
};

inline object none() { return object(); }

class python_error : public std::runtime_error {
public:
    python_error() : std::runtime_error("interrupted") {}
};

template <typename T>
struct is_ndarray : std::false_type {};
template <typename... A>
struct is_ndarray<ndarray<A...>> : std::true_type {};

template <typename T>
T cast(const object& o) {
    if constexpr (is_ndarray<T>::value) {
        if (o.kind() != object::Kind::Array)
            throw std::runtime_error("nbshim: cast to ndarray from a non-array object");
        using S = typename T::Scalar;
        if constexpr (!std::is_void_v<S>) {
            if (o.a_.dt != dtype<S>())
                throw std::runtime_error("nbshim: ndarray dtype mismatch in cast");
        }
        return T(o.a_);
    } else if constexpr (std::is_integral_v<T>) {
        if (o.kind() != object::Kind::Int)
            throw std::runtime_error("nbshim: cast to integer from a non-integer object");
        return (T)o.u_ ? (T)o.u_ : (T)o.i_;
    } else if constexpr (std::is_floating_point_v<T>) {
        if (o.kind() == object::Kind::Float) return (T)o.f_;
        if (o.kind() == object::Kind::Int) return (T)o.i_;
        throw std::runtime_error("nbshim: cast to float from a non-number object");
    } else {
        static_assert(sizeof(T) == 0, "nbshim: unsupported cast");
    }
}

class tuple {
public:
    std::vector<object> items;
    object operator[](size_t i) const { return items.at(i); }
    size_t size() const { return items.size(); }
};

template <typename... A>
tuple make_tuple(A&&... a) {
    tuple t;
    (t.items.push_back(object(std::forward<A>(a))), ...);
    return t;
}

class dict {
public:
    struct proxy {
        template <typename V> proxy& operator=(V&&) { return *this; }
    };
    proxy operator[](const char*) { return proxy{}; }
};

struct gil_scoped_acquire {};
struct gil_scoped_release {};

struct arg {
    explicit arg(const char*) {}
    template <typename V> arg& operator=(V&&) { return *this; }
};

class module_ {
public:
    std::string& doc() { return doc_; }
    template <typename... A> module_& def(A&&...) { return *this; }
private:
    std::string doc_;
};

}  // namespace nanobind

#define NB_MODULE(name, m) \
    [[maybe_unused]] static void nbshim_module_init_##name(::nanobind::module_& m)
