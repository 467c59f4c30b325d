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
    template <typename P, typename O>
    ndarray(P* ptr, std::initializer_list<size_t> shp, const O& owner_object)
        : ndarray(ptr, shp, capsule()) {
        (void)owner_object;  // caller keeps the owning object alive
    }
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
    // Element strides of a dense array: column-major when the type says
    // f_contig, row-major otherwise.
    int64_t stride(size_t i) const {
        int64_t st = 1;
        if (is_f_order()) {
            for (size_t k = 0; k < i; ++k) st *= (int64_t)d.shape[k];
        } else {
            for (size_t k = i + 1; k < d.ndim; ++k) st *= (int64_t)d.shape[k];
        }
        return st;
    }
    template <typename... I, typename S = Scalar>
    S& operator()(I... idx) const {
        const size_t ix[] = {(size_t)idx...};
        size_t off = 0;
        for (size_t k = 0; k < sizeof...(I); ++k) off += ix[k] * (size_t)stride(k);
        return data()[off];
    }
    static constexpr bool is_f_order() { return (std::is_same_v<Args, struct f_contig> || ...); }
};

template <typename T>
struct is_ndarray : std::false_type {};
template <typename... A>
struct is_ndarray<ndarray<A...>> : std::true_type {};

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
    template <typename V, std::enable_if_t<std::is_integral_v<V>, int> = 0>
    object(V v) : i_((int64_t)v), u_((uint64_t)v), kind_(Kind::Int) {}
    template <typename V, std::enable_if_t<std::is_floating_point_v<V>, int> = 0>
    object(V v) : f_((double)v), kind_(Kind::Float) {}
    template <typename V, std::enable_if_t<std::is_class_v<std::decay_t<V>> &&
                                             !is_ndarray<std::decay_t<V>>::value &&
                                             !std::is_same_v<std::decay_t<V>, object> &&
                                             !std::is_same_v<std::decay_t<V>, std::string>, int> = 0>
    object(V&&) : kind_(Kind::None) {}  // list / dict / tuple results are not inspected
    object(const char*) : kind_(Kind::Str) {}
    object(const std::string&) : kind_(Kind::Str) {}
    object attr(const char*) const { return object(); }
    template <typename... A> object operator()(A&&...) const { return object(); }

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

enum class rv_policy { automatic, automatic_reference, take_ownership, copy, move, reference,
                       reference_internal, none };

// C++ value -> object (the inverse direction of cast<T>(object)).
template <typename V>
object cast(V&& v, rv_policy = rv_policy::automatic) {
    if constexpr (is_ndarray<std::decay_t<V>>::value) return object(v);
    else if constexpr (std::is_arithmetic_v<std::decay_t<V>>) return object(v);
    else return object();
}

template <typename T> size_t len(const T& v) { return v.size(); }

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
        object value;
        template <typename V> proxy& operator=(V&&) { return *this; }
        operator const object&() const { return value; }
    };
    proxy operator[](const char*) { return proxy{}; }
    proxy operator[](const char*) const { return proxy{}; }
    proxy operator[](const std::string&) const { return proxy{}; }
    bool contains(const char*) const { return false; }
    size_t size() const { return 0; }
};

class list {
public:
    std::vector<object> items;
    list() = default;
    template <typename V> void append(V&& v) { items.push_back(object(std::forward<V>(v))); }
    size_t size() const { return items.size(); }
    object operator[](size_t i) const { return items.at(i); }
};

template <typename... A> struct init {};
struct kw_only {};

struct gil_scoped_acquire {};
struct gil_scoped_release {};

struct arg {
    explicit arg(const char*) {}
    template <typename V> arg& operator=(V&&) { return *this; }
    arg& noconvert(bool = true) { return *this; }
    arg& none(bool = true) { return *this; }
};

class module_ {
public:
    std::string& doc() { return doc_; }
    template <typename... A> module_& def(A&&...) { return *this; }
    object attr(const char*) const { return object(); }
    static module_ import_(const char*) { return module_(); }
private:
    std::string doc_;
};

// Class registration is parsed but never run (NB_MODULE bodies are templates).
template <typename T, typename... Extra>
class class_ {
public:
    template <typename... A> class_(A&&...) {}
    template <typename... A> class_& def(A&&...) { return *this; }
    template <typename... A> class_& def_prop_ro(A&&...) { return *this; }
    template <typename... A> class_& def_static(A&&...) { return *this; }
    template <typename... A> class_& def_ro(A&&...) { return *this; }
};

}  // namespace nanobind

// The module body is a template that is never instantiated: it is parsed, but
// registration calls on the dependent module object are not resolved.
#define NB_MODULE(name, m) \
    template <typename NbShimModuleT> \
    [[maybe_unused]] static void nbshim_module_init_##name(NbShimModuleT& m)
