// A subset of the xtensor 0.25 API (https://github.com/xtensor-stack/xtensor,
// BSD-3-Clause; this file restates its documented semantics and shares no code
// with it): the containers, views, builders, element-wise operations,
// reducers and .npy writer that the XFDTD API and its programs use.
//
// Design: every operation evaluates eagerly into a dense row-major container
// (xtensor evaluates lazily; the element values are the same because each
// element is computed by the same sequence of scalar operations).  Assigning
// to a view evaluates the right-hand side into a temporary first, so
// overlapping views of one array assign as xtensor's temporary-based
// assignment does.  Shapes broadcast as in NumPy.
//
// Containers: xt::xarray<T> (rank fixed at run time), xt::xtensor<T, N>
// (rank N), xt::xtensor_fixed<T, xt::xshape<I...>>.  Views: xt::view(e,
// slices...) with xt::range(start, stop[, step]), integer indices (drop the
// axis), xt::all(); a view is writable and can be viewed again.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <functional>
#include <initializer_list>
#include <iostream>
#include <iterator>
#include <limits>
#include <memory>
#include <numeric>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace xt {

// Shapes and strides: a vector-like sequence with inline storage (ranks up to
// 8), so that small arrays and per-element temporaries allocate no heap blocks
// for them.
template <class T>
class svector {
 public:
  static constexpr std::size_t cap = 8;
  using value_type = T;
  using size_type = std::size_t;
  using iterator = T*;
  using const_iterator = const T*;
  svector() = default;
  explicit svector(std::size_t n, const T& v = T()) { resize(n, v); }
  svector(std::initializer_list<T> l) { assign(l.begin(), l.end()); }
  template <class It, class = decltype(*std::declval<It>())>
  svector(It a, It b) {
    assign(a, b);
  }
  template <class U, std::size_t N>
  svector(const std::array<U, N>& a) {
    assign(a.begin(), a.end());
  }
  // Integer sequences only: a vector of values is not a shape.
  template <class U, std::enable_if_t<std::is_integral_v<U>, int> = 0>
  svector(const std::vector<U>& v) {
    assign(v.begin(), v.end());
  }
  template <class It>
  void assign(It a, It b) {
    n_ = 0;
    for (; a != b; ++a) push_back((T)*a);
  }
  std::size_t size() const { return n_; }
  bool empty() const { return n_ == 0; }
  T* data() { return v_; }
  const T* data() const { return v_; }
  T* begin() { return v_; }
  T* end() { return v_ + n_; }
  const T* begin() const { return v_; }
  const T* end() const { return v_ + n_; }
  T& operator[](std::size_t i) { return v_[i]; }
  const T& operator[](std::size_t i) const { return v_[i]; }
  T& front() { return v_[0]; }
  const T& front() const { return v_[0]; }
  T& back() { return v_[n_ - 1]; }
  const T& back() const { return v_[n_ - 1]; }
  void push_back(const T& x) {
    if (n_ == cap) throw std::length_error("xt: rank above 8");
    v_[n_++] = x;
  }
  void resize(std::size_t n, const T& x = T()) {
    if (n > cap) throw std::length_error("xt: rank above 8");
    for (std::size_t i = n_; i < n; ++i) v_[i] = x;
    n_ = n;
  }
  T* insert(T* pos, const T& x) {
    const std::size_t at = (std::size_t)(pos - v_);
    push_back(x);
    for (std::size_t i = n_ - 1; i > at; --i) v_[i] = v_[i - 1];
    v_[at] = x;
    return v_ + at;
  }
  T* erase(T* pos) {
    for (T* p = pos; p + 1 < v_ + n_; ++p) *p = p[1];
    --n_;
    return pos;
  }
  operator std::vector<T>() const { return std::vector<T>(begin(), end()); }
  friend bool operator==(const svector& a, const svector& b) {
    return a.n_ == b.n_ && std::equal(a.begin(), a.end(), b.begin());
  }
  friend bool operator!=(const svector& a, const svector& b) { return !(a == b); }

 private:
  T v_[cap] = {};
  std::size_t n_ = 0;
};

using shape_type = svector<std::size_t>;
using strides_type = svector<std::ptrdiff_t>;

template <class T>
class xarray;
template <class T, std::size_t N>
class xtensor;
template <class T>
class xview;
template <std::size_t... I>
struct xshape {};
template <class T, class S>
class xtensor_fixed;

// ---------------------------------------------------------------- traits
template <class E>
struct is_xexpr : std::false_type {};
template <class T>
struct is_xexpr<xarray<T>> : std::true_type {};
template <class T, std::size_t N>
struct is_xexpr<xtensor<T, N>> : std::true_type {};
template <class T>
struct is_xexpr<xview<T>> : std::true_type {};
template <class T, std::size_t... I>
struct is_xexpr<xtensor_fixed<T, xshape<I...>>> : std::true_type {};
template <class E>
inline constexpr bool is_xexpr_v = is_xexpr<std::decay_t<E>>::value;

template <class T>
struct is_complex : std::false_type {};
template <class T>
struct is_complex<std::complex<T>> : std::true_type {};
template <class S>
inline constexpr bool is_scalar_v =
    std::is_arithmetic_v<std::decay_t<S>> || is_complex<std::decay_t<S>>::value;

namespace detail {

inline std::size_t prod(const shape_type& s) {
  std::size_t n = 1;
  for (std::size_t v : s) n *= v;
  return n;
}

inline strides_type row_major(const shape_type& s) {
  strides_type st(s.size());
  std::ptrdiff_t acc = 1;
  for (std::size_t d = s.size(); d-- > 0;) {
    st[d] = s[d] == 1 ? 0 : acc;  // length-1 axes broadcast (stride 0), as in xtensor
    acc *= (std::ptrdiff_t)s[d];
  }
  return st;
}

// Calls f(offset) for every element of (shape, strides) in row-major order.
template <class F>
void for_each_offset(const shape_type& shape, const strides_type& st, std::ptrdiff_t base, F&& f) {
  const std::size_t n = prod(shape);
  if (n == 0) return;
  const std::size_t r = shape.size();
  if (r == 0) {
    f(base);
    return;
  }
  std::size_t idx[svector<std::size_t>::cap] = {};
  std::ptrdiff_t off = base;
  const std::size_t inner = shape[r - 1];
  const std::ptrdiff_t ist = st[r - 1];
  for (std::size_t done = 0; done < n; done += inner) {
    std::ptrdiff_t o = off;
    for (std::size_t k = 0; k < inner; ++k, o += ist) f(o);
    // advance the outer indices
    for (std::size_t d = r - 1; d-- > 0;) {
      if (++idx[d] < shape[d]) {
        off += st[d];
        break;
      }
      off -= (std::ptrdiff_t)(shape[d] - 1) * st[d];
      idx[d] = 0;
    }
  }
}

inline shape_type broadcast_shapes(const shape_type& a, const shape_type& b) {
  const std::size_t r = std::max(a.size(), b.size());
  shape_type out(r);
  for (std::size_t d = 0; d < r; ++d) {
    const std::size_t x = d + a.size() >= r ? a[d + a.size() - r] : 1;
    const std::size_t y = d + b.size() >= r ? b[d + b.size() - r] : 1;
    if (x != y && x != 1 && y != 1) throw std::runtime_error("xt: shapes do not broadcast");
    out[d] = x == 1 ? y : x;
  }
  return out;
}

// Strides of an array of shape `s` (strides `st`) broadcast to shape `to`.
inline strides_type broadcast_strides(const shape_type& s, const strides_type& st,
                                      const shape_type& to) {
  strides_type out(to.size(), 0);
  const std::size_t off = to.size() - s.size();
  for (std::size_t d = 0; d < s.size(); ++d) out[off + d] = s[d] == 1 ? 0 : st[d];
  return out;
}

// Element storage: up to 4 numeric elements inline (small vectors such as a
// 3-component coordinate), otherwise one heap block.
template <class T>
struct buffer {
  static constexpr std::size_t inline_cap =
      (std::is_arithmetic_v<T> || is_complex<T>::value) ? 4 : 0;
  std::unique_ptr<T[]> heap;
  T small[inline_cap > 0 ? inline_cap : 1] = {};
  T* p = nullptr;
  std::size_t n = 0;
  buffer() = default;
  explicit buffer(std::size_t m) : n(m) {
    if (m == 0) return;
    if (m <= inline_cap) {
      for (std::size_t i = 0; i < m; ++i) small[i] = T();
      p = small;
    } else {
      heap.reset(new T[m]());
      p = heap.get();
    }
  }
  buffer(const buffer& o) : buffer(o.n) { std::copy(o.p, o.p + o.n, p); }
  buffer(buffer&& o) noexcept { steal(std::move(o)); }
  buffer& operator=(const buffer& o) {
    if (this != &o) {
      buffer t(o);
      steal(std::move(t));
    }
    return *this;
  }
  buffer& operator=(buffer&& o) noexcept {
    if (this != &o) steal(std::move(o));
    return *this;
  }
  T* get() const { return p; }

 private:
  void steal(buffer&& o) {
    n = o.n;
    if (o.p == o.small) {
      heap.reset();
      for (std::size_t i = 0; i < n; ++i) small[i] = std::move(o.small[i]);
      p = n ? small : nullptr;
    } else {
      heap = std::move(o.heap);
      p = heap.get();
    }
    o.p = nullptr;
    o.n = 0;
  }
};

}  // namespace detail

// ---------------------------------------------------------------- slices
// xt::placeholders::_ stands for an open end of a range; programs written for
// xtensor use it unqualified, so it is also declared at global scope below.
namespace placeholders {
struct xtuph {};
inline constexpr xtuph _{};
}  // namespace placeholders

struct xrange_t {
  static constexpr long long open = std::numeric_limits<long long>::min();
  long long start, stop, step;
};
namespace detail {
template <class A>
long long range_bound(const A& a) {
  if constexpr (std::is_same_v<A, placeholders::xtuph>) return xrange_t::open;
  else return (long long)a;
}
}  // namespace detail
template <class A, class B>
xrange_t range(A a, B b) {
  return {detail::range_bound(a), detail::range_bound(b), 1};
}
template <class A, class B, class C>
xrange_t range(A a, B b, C c) {
  return {detail::range_bound(a), detail::range_bound(b), (long long)c};
}
struct xall_t {};
inline xall_t all() { return {}; }

// ---------------------------------------------------------------- dense storage
template <class T>
class xdense {
 public:
  using value_type = T;
  using size_type = std::size_t;
  using reference = T&;
  using const_reference = const T&;
  using pointer = T*;
  using iterator = T*;
  using const_iterator = const T*;
  using shape_type = xt::shape_type;

  xdense() = default;
  explicit xdense(const shape_type& s) { reset(s); }
  xdense(const shape_type& s, const T& v) {
    reset(s);
    std::fill(begin(), end(), v);
  }

  const shape_type& shape() const { return shape_; }
  std::size_t shape(std::size_t d) const { return shape_[d]; }
  const strides_type& strides() const { return strides_; }
  std::size_t dimension() const { return shape_.size(); }
  std::size_t size() const { return buf_.n; }
  T* data() { return buf_.get(); }
  const T* data() const { return buf_.get(); }
  std::ptrdiff_t data_offset() const { return 0; }
  T* begin() { return data(); }
  T* end() { return data() + size(); }
  const T* begin() const { return data(); }
  const T* end() const { return data() + size(); }
  const T* cbegin() const { return data(); }
  const T* cend() const { return data() + size(); }
  T& front() { return data()[0]; }
  const T& front() const { return data()[0]; }
  T& back() { return data()[size() - 1]; }
  const T& back() const { return data()[size() - 1]; }
  T& flat(std::size_t i) { return data()[i]; }
  const T& flat(std::size_t i) const { return data()[i]; }
  T& operator[](std::size_t i) { return data()[i]; }
  const T& operator[](std::size_t i) const { return data()[i]; }
  void fill(const T& v) { std::fill(begin(), end(), v); }

  template <class... I>
  T& operator()(I... idx) {
    return data()[offset(idx...)];
  }
  template <class... I>
  const T& operator()(I... idx) const {
    return data()[offset(idx...)];
  }
  template <class... I>
  T& at(I... idx) {
    check(idx...);
    return data()[offset(idx...)];
  }
  template <class... I>
  const T& at(I... idx) const {
    check(idx...);
    return data()[offset(idx...)];
  }
  T& element(const std::vector<std::size_t>& idx) {
    std::ptrdiff_t o = 0;
    for (std::size_t d = 0; d < idx.size(); ++d) o += (std::ptrdiff_t)idx[d] * full_[d];
    return data()[o];
  }

  template <class S>
  void resize(const S& s) {
    shape_type ns(std::begin(s), std::end(s));
    if (ns == shape_ && size() == detail::prod(ns)) return;
    reset(ns);
  }
  void resize(std::initializer_list<std::size_t> s) { resize(shape_type(s)); }
  template <class S>
  void reshape(const S& s) {
    shape_type ns(std::begin(s), std::end(s));
    if (detail::prod(ns) != size()) throw std::runtime_error("xt: reshape changes the size");
    shape_ = ns;
    strides_ = detail::row_major(ns);
    full_ = full_strides(ns);
  }
  void reshape(std::initializer_list<std::size_t> s) { reshape(shape_type(s)); }

 protected:
  void reset(const shape_type& s) {
    shape_ = s;
    strides_ = detail::row_major(s);
    full_ = full_strides(s);
    buf_ = detail::buffer<T>(detail::prod(s));
  }
  void take(xdense&& o) {
    shape_ = std::move(o.shape_);
    strides_ = std::move(o.strides_);
    full_ = std::move(o.full_);
    buf_ = std::move(o.buf_);
  }
  static strides_type full_strides(const shape_type& s) {
    strides_type st(s.size());
    std::ptrdiff_t acc = 1;
    for (std::size_t d = s.size(); d-- > 0;) {
      st[d] = acc;
      acc *= (std::ptrdiff_t)s[d];
    }
    return st;
  }
  // xtensor's indexing rule: with more indices than dimensions the leading
  // ones are dropped; with fewer, they address the trailing dimensions.
  template <class... I>
  std::ptrdiff_t offset(I... idx) const {
    constexpr std::size_t n = sizeof...(I);
    if constexpr (n == 0) {
      return 0;
    } else {
      const std::ptrdiff_t v[n] = {(std::ptrdiff_t)idx...};
      const std::size_t r = full_.size();
      std::ptrdiff_t o = 0;
      if (n >= r) {
        for (std::size_t d = 0; d < r; ++d) o += v[n - r + d] * full_[d];
      } else {
        for (std::size_t d = 0; d < n; ++d) o += v[d] * full_[r - n + d];
      }
      return o;
    }
  }
  template <class... I>
  void check(I... idx) const {
    constexpr std::size_t n = sizeof...(I);
    const std::size_t v[n > 0 ? n : 1] = {(std::size_t)idx...};
    const std::size_t r = shape_.size();
    for (std::size_t d = 0; d < std::min(n, r); ++d)
      if (v[n >= r ? n - r + d : d] >= shape_[n >= r ? d : r - n + d])
        throw std::out_of_range("xt: index out of range");
  }

  shape_type shape_;
  strides_type strides_;  // broadcast strides (0 on length-1 axes)
  strides_type full_;     // plain row-major strides (element access)
  detail::buffer<T> buf_;
};

// Evaluation of any expression into a dense array (declared here, defined
// after the containers).
template <class E>
auto eval(const E& e);

namespace detail {
template <class E>
using value_t = typename std::decay_t<E>::value_type;

// Copies expression e (of shape `to` after broadcasting) into dst, row-major.
template <class E, class T>
void copy_broadcast(const E& e, const shape_type& to, T* dst) {
  const strides_type st = broadcast_strides(e.shape(), e.strides(), to);
  const auto* src = e.data();
  std::size_t k = 0;
  for_each_offset(to, st, e.data_offset(), [&](std::ptrdiff_t o) { dst[k++] = (T)src[o]; });
}
}  // namespace detail

// ---------------------------------------------------------------- xarray
template <class T>
class xarray : public xdense<T> {
 public:
  using base = xdense<T>;
  using base::base;
  xarray() { this->reset(shape_type{}); }
  xarray(const xarray&) = default;
  xarray(xarray&&) noexcept = default;
  xarray& operator=(const xarray&) = default;
  xarray& operator=(xarray&&) noexcept = default;
  xarray(std::initializer_list<T> l) {
    this->reset(shape_type{l.size()});
    std::copy(l.begin(), l.end(), this->begin());
  }
  xarray(std::initializer_list<std::initializer_list<T>> l) {
    const std::size_t r = l.size(), c = r ? l.begin()->size() : 0;
    this->reset(shape_type{r, c});
    std::size_t k = 0;
    for (const auto& row : l)
      for (const auto& v : row) this->data()[k++] = v;
  }
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xarray(const E& e) {
    this->reset(e.shape());
    detail::copy_broadcast(e, e.shape(), this->data());
  }
  template <class U, std::size_t N>
  xarray(xtensor<U, N>&& e);
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xarray& operator=(const E& e) {
    xarray t(e);
    *this = std::move(t);
    return *this;
  }
  xarray& operator=(const T& v) {
    this->fill(v);
    return *this;
  }
  static xarray from_shape(const shape_type& s) { return xarray(s); }
  template <class S>
  static xarray from_shape(const S& s) {
    return xarray(shape_type(std::begin(s), std::end(s)));
  }
  void take_from(xdense<T>&& o) { this->take(std::move(o)); }
};

// ---------------------------------------------------------------- xtensor
template <class T, std::size_t N>
class xtensor : public xdense<T> {
 public:
  using base = xdense<T>;
  using shape_type = xt::shape_type;
  xtensor() { this->reset(shape_type(N, 0)); }
  xtensor(const xtensor&) = default;
  xtensor(xtensor&&) noexcept = default;
  xtensor& operator=(const xtensor&) = default;
  xtensor& operator=(xtensor&&) noexcept = default;
  explicit xtensor(const shape_type& s) : base(s) { rank_check(); }
  xtensor(const shape_type& s, const T& v) : base(s, v) { rank_check(); }
  template <std::size_t M = N, std::enable_if_t<M == 1, int> = 0>
  xtensor(std::initializer_list<T> l) {
    this->reset(shape_type{l.size()});
    std::copy(l.begin(), l.end(), this->begin());
  }
  template <std::size_t M = N, std::enable_if_t<M == 2, int> = 0>
  xtensor(std::initializer_list<std::initializer_list<T>> l) {
    const std::size_t r = l.size(), c = r ? l.begin()->size() : 0;
    this->reset(shape_type{r, c});
    std::size_t k = 0;
    for (const auto& row : l)
      for (const auto& v : row) this->data()[k++] = v;
  }
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xtensor(const E& e) {
    this->reset(e.shape());
    rank_check();
    detail::copy_broadcast(e, e.shape(), this->data());
  }
  xtensor(xarray<T>&& a) {  // take the buffer
    this->take_from(std::move(a));
    rank_check();
  }
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xtensor& operator=(const E& e) {
    xtensor t(e);
    *this = std::move(t);
    return *this;
  }
  xtensor& operator=(xarray<T>&& a) {
    this->take_from(std::move(a));
    rank_check();
    return *this;
  }
  xtensor& operator=(const T& v) {
    this->fill(v);
    return *this;
  }
  static xtensor from_shape(const shape_type& s) { return xtensor(s); }
  template <class S>
  static xtensor from_shape(const S& s) {
    return xtensor(shape_type(std::begin(s), std::end(s)));
  }
  static xtensor from_shape(std::initializer_list<std::size_t> s) { return xtensor(shape_type(s)); }
  void take_from(xdense<T>&& o) { this->take(std::move(o)); }

  // Element access with the rank known at compile time (one multiply-add per
  // index, no run-time rank loop), as xtensor's fixed-rank containers do.
  template <class... I>
  T& operator()(I... idx) {
    if constexpr (sizeof...(I) == N) return this->data()[fixed_offset(idx...)];
    else return base::operator()(idx...);
  }
  template <class... I>
  const T& operator()(I... idx) const {
    if constexpr (sizeof...(I) == N) return this->data()[fixed_offset(idx...)];
    else return base::operator()(idx...);
  }

 private:
  template <class... I>
  std::ptrdiff_t fixed_offset(I... idx) const {
    const std::ptrdiff_t v[N > 0 ? N : 1] = {(std::ptrdiff_t)idx...};
    const std::ptrdiff_t* st = this->full_.data();
    std::ptrdiff_t o = 0;
#pragma GCC unroll 8
    for (std::size_t d = 0; d < N; ++d) o += v[d] * st[d];
    return o;
  }
  void rank_check() const {
    if (this->shape_.size() != N) throw std::runtime_error("xt::xtensor: rank mismatch");
  }
};

template <class T>
template <class U, std::size_t N>
xarray<T>::xarray(xtensor<U, N>&& e) {
  if constexpr (std::is_same_v<T, U>) {
    this->take(std::move(static_cast<xdense<U>&>(e)));
  } else {
    this->reset(e.shape());
    detail::copy_broadcast(e, e.shape(), this->data());
  }
}

// ---------------------------------------------------------------- xtensor_fixed
template <class T, std::size_t... I>
class xtensor_fixed<T, xshape<I...>> : public xdense<T> {
 public:
  xtensor_fixed() { this->reset(shape_type{I...}); }
  xtensor_fixed(const xtensor_fixed&) = default;
  xtensor_fixed(xtensor_fixed&&) noexcept = default;
  xtensor_fixed& operator=(const xtensor_fixed&) = default;
  xtensor_fixed& operator=(xtensor_fixed&&) noexcept = default;
  xtensor_fixed(std::initializer_list<T> l) {
    this->reset(shape_type{I...});
    std::copy(l.begin(), l.end(), this->begin());
  }
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xtensor_fixed(const E& e) {
    this->reset(shape_type{I...});
    detail::copy_broadcast(e, this->shape_, this->data());
  }
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xtensor_fixed& operator=(const E& e) {
    xtensor_fixed t(e);
    *this = std::move(t);
    return *this;
  }
};

// ---------------------------------------------------------------- xview
template <class T>
class xview {
 public:
  using value_type = std::remove_const_t<T>;
  using size_type = std::size_t;
  using shape_type = xt::shape_type;

  xview(T* base, std::ptrdiff_t off, shape_type shape, strides_type st,
        std::shared_ptr<void> keep = nullptr)
      : base_(base), off_(off), shape_(std::move(shape)), st_(std::move(st)),
        keep_(std::move(keep)) {}
  xview(const xview&) = default;

  const shape_type& shape() const { return shape_; }
  std::size_t shape(std::size_t d) const { return shape_[d]; }
  const strides_type& strides() const { return st_; }
  std::size_t dimension() const { return shape_.size(); }
  std::size_t size() const { return detail::prod(shape_); }
  T* data() const { return base_; }
  std::ptrdiff_t data_offset() const { return off_; }

  template <class... I>
  T& operator()(I... idx) const {
    constexpr std::size_t n = sizeof...(I);
    if constexpr (n == 0) {
      return base_[off_];
    } else {
      const std::ptrdiff_t v[n] = {(std::ptrdiff_t)idx...};
      const std::size_t r = st_.size();
      std::ptrdiff_t o = off_;
      if (n >= r) {
        for (std::size_t d = 0; d < r; ++d) o += v[n - r + d] * st_[d];
      } else {
        for (std::size_t d = 0; d < n; ++d) o += v[d] * st_[r - n + d];
      }
      return base_[o];
    }
  }
  T& flat(std::size_t i) const {
    std::ptrdiff_t o = off_;
    for (std::size_t d = shape_.size(); d-- > 0;) {
      o += (std::ptrdiff_t)(i % shape_[d]) * st_[d];
      i /= shape_[d];
    }
    return base_[o];
  }
  T& operator[](std::size_t i) const { return flat(i); }
  T& front() const { return flat(0); }
  T& back() const { return flat(size() - 1); }

  class iterator {
   public:
    using iterator_category = std::forward_iterator_tag;
    using value_type = std::remove_const_t<T>;
    using difference_type = std::ptrdiff_t;
    using pointer = T*;
    using reference = T&;
    iterator(const xview* v, std::size_t i) : v_(v), i_(i) {}
    T& operator*() const { return v_->flat(i_); }
    iterator& operator++() {
      ++i_;
      return *this;
    }
    iterator operator++(int) {
      iterator t = *this;
      ++i_;
      return t;
    }
    bool operator==(const iterator& o) const { return i_ == o.i_; }
    bool operator!=(const iterator& o) const { return i_ != o.i_; }

   private:
    const xview* v_;
    std::size_t i_;
  };
  iterator begin() const { return iterator(this, 0); }
  iterator end() const { return iterator(this, size()); }

  // Assignment writes the elements (evaluating the right-hand side first).
  xview& operator=(const xview& o) { return assign(o); }
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
  xview& operator=(const E& e) {
    return assign(e);
  }
  template <class S, std::enable_if_t<is_scalar_v<S>, int> = 0>
  xview& operator=(const S& s) {
    detail::for_each_offset(shape_, st_, off_, [&](std::ptrdiff_t o) { base_[o] = (value_type)s; });
    return *this;
  }
  template <class E>
  xview& operator+=(const E& e) {
    return compound(e, std::plus<>());
  }
  template <class E>
  xview& operator-=(const E& e) {
    return compound(e, std::minus<>());
  }
  template <class E>
  xview& operator*=(const E& e) {
    return compound(e, std::multiplies<>());
  }
  template <class E>
  xview& operator/=(const E& e) {
    return compound(e, std::divides<>());
  }

 private:
  template <class E>
  xview& assign(const E& e) {
    const xarray<value_type> t(e);
    const strides_type sst = detail::broadcast_strides(t.shape(), t.strides(), shape_);
    std::vector<std::ptrdiff_t> src;
    src.reserve(size());
    detail::for_each_offset(shape_, sst, 0, [&](std::ptrdiff_t o) { src.push_back(o); });
    std::size_t k = 0;
    detail::for_each_offset(shape_, st_, off_,
                            [&](std::ptrdiff_t o) { base_[o] = t.data()[src[k++]]; });
    return *this;
  }
  template <class E, class F>
  xview& compound(const E& e, F f) {
    if constexpr (is_scalar_v<E>) {
      detail::for_each_offset(shape_, st_, off_,
                              [&](std::ptrdiff_t o) { base_[o] = (value_type)f(base_[o], e); });
    } else {
      const xarray<value_type> t(e);
      const strides_type sst = detail::broadcast_strides(t.shape(), t.strides(), shape_);
      std::vector<std::ptrdiff_t> src;
      src.reserve(size());
      detail::for_each_offset(shape_, sst, 0, [&](std::ptrdiff_t o) { src.push_back(o); });
      std::size_t k = 0;
      detail::for_each_offset(shape_, st_, off_, [&](std::ptrdiff_t o) {
        base_[o] = (value_type)f(base_[o], t.data()[src[k++]]);
      });
    }
    return *this;
  }

  T* base_;
  std::ptrdiff_t off_;
  shape_type shape_;
  strides_type st_;
  std::shared_ptr<void> keep_;
};

namespace detail {

inline void apply_slice(const shape_type& s, const strides_type& st, std::size_t& d,
                        std::ptrdiff_t& off, shape_type& ns, strides_type& nst,
                        const xrange_t& r) {
  const long long n = (long long)s[d];
  const long long step = r.step == 0 ? 1 : r.step;
  long long a = r.start == xrange_t::open ? (step > 0 ? 0 : n - 1) : r.start;
  long long b = r.stop == xrange_t::open ? (step > 0 ? n : -n - 1) : r.stop;
  if (a < 0) a += n;
  if (b < 0) b += n;
  a = std::clamp(a, step > 0 ? 0LL : -1LL, step > 0 ? n : n - 1);
  b = std::clamp(b, -1LL, n);
  long long len = step > 0 ? (b > a ? (b - a + step - 1) / step : 0)
                           : (a > b ? (a - b + (-step) - 1) / (-step) : 0);
  off += (std::ptrdiff_t)a * st[d];
  ns.push_back((std::size_t)len);
  nst.push_back((std::ptrdiff_t)step * st[d]);
  ++d;
}
inline void apply_slice(const shape_type& s, const strides_type& st, std::size_t& d,
                        std::ptrdiff_t&, shape_type& ns, strides_type& nst, const xall_t&) {
  ns.push_back(s[d]);
  nst.push_back(st[d]);
  ++d;
}
template <class I, std::enable_if_t<std::is_integral_v<I>, int> = 0>
void apply_slice(const shape_type&, const strides_type& st, std::size_t& d, std::ptrdiff_t& off,
                 shape_type&, strides_type&, I i) {
  off += (std::ptrdiff_t)i * st[d];
  ++d;
}

template <class T, class... S>
xview<T> make_view(T* base, std::ptrdiff_t off, const shape_type& s, const strides_type& st,
                   std::shared_ptr<void> keep, const S&... sl) {
  shape_type ns;
  strides_type nst;
  std::size_t d = 0;
  (apply_slice(s, st, d, off, ns, nst, sl), ...);
  for (; d < s.size(); ++d) {
    ns.push_back(s[d]);
    nst.push_back(st[d]);
  }
  return xview<T>(base, off, std::move(ns), std::move(nst), std::move(keep));
}

// Plain (non-broadcast) strides of a dense container.
template <class T>
strides_type plain_strides(const xdense<T>& c) {
  strides_type st(c.shape().size());
  std::ptrdiff_t acc = 1;
  for (std::size_t d = c.shape().size(); d-- > 0;) {
    st[d] = acc;
    acc *= (std::ptrdiff_t)c.shape()[d];
  }
  return st;
}

}  // namespace detail

template <class T, class... S>
xview<T> view(xdense<T>& c, const S&... sl) {
  return detail::make_view<T>(c.data(), 0, c.shape(), detail::plain_strides(c), nullptr, sl...);
}
template <class T, class... S>
xview<const T> view(const xdense<T>& c, const S&... sl) {
  return detail::make_view<const T>(c.data(), 0, c.shape(), detail::plain_strides(c), nullptr,
                                    sl...);
}
template <class T, class... S>
xview<T> view(const xview<T>& v, const S&... sl) {
  return detail::make_view<T>(v.data(), v.data_offset(), v.shape(), v.strides(), nullptr, sl...);
}
// A view of a temporary keeps it alive.
template <class C, class... S,
          std::enable_if_t<!std::is_lvalue_reference_v<C> && is_xexpr_v<C> &&
                               !std::is_same_v<std::decay_t<C>,
                                               xview<typename std::decay_t<C>::value_type>> &&
                               !std::is_same_v<std::decay_t<C>,
                                               xview<const typename std::decay_t<C>::value_type>>,
                           int> = 0>
auto view(C&& c, const S&... sl) {
  using T = typename std::decay_t<C>::value_type;
  auto keep = std::make_shared<xarray<T>>(std::forward<C>(c));
  return detail::make_view<T>(keep->data(), 0, keep->shape(), detail::plain_strides(*keep), keep,
                              sl...);
}

// ---------------------------------------------------------------- evaluation
template <class E>
auto eval(const E& e) {
  using T = detail::value_t<E>;
  return xarray<T>(e);
}

namespace detail {

template <class S>
struct scalar_ref {
  const S& s;
};

template <class E>
decltype(auto) operand_value(const E& e, std::size_t) {
  return e;
}

// Element-wise map of one expression.
template <class F, class E>
auto map1(F f, const E& e) {
  using V = value_t<E>;
  using R = std::decay_t<decltype(f(std::declval<V>()))>;
  const shape_type s = e.shape();
  xarray<R> out{xarray<R>::from_shape(s)};
  if constexpr (std::is_base_of_v<xdense<V>, std::decay_t<E>>) {
    const V* a = e.data();
    for (std::size_t i = 0; i < out.size(); ++i) out.data()[i] = f(a[i]);
  } else {
    const auto* src = e.data();
    std::size_t k = 0;
    for_each_offset(s, e.strides(), e.data_offset(),
                    [&](std::ptrdiff_t o) { out.data()[k++] = f(src[o]); });
  }
  return out;
}

// Element-wise map of two operands (expressions or scalars), broadcast.
template <class F, class A, class B>
auto map2(F f, const A& a, const B& b) {
  if constexpr (is_scalar_v<A>) {
    return map1([&](const auto& y) { return f(a, y); }, b);
  } else if constexpr (is_scalar_v<B>) {
    return map1([&](const auto& x) { return f(x, b); }, a);
  } else {
    using VA = value_t<A>;
    using VB = value_t<B>;
    using R = std::decay_t<decltype(f(std::declval<VA>(), std::declval<VB>()))>;
    const shape_type s = broadcast_shapes(a.shape(), b.shape());
    xarray<R> out{xarray<R>::from_shape(s)};
    const bool dense_a = std::is_base_of_v<xdense<VA>, std::decay_t<A>> && a.shape() == s;
    const bool dense_b = std::is_base_of_v<xdense<VB>, std::decay_t<B>> && b.shape() == s;
    if (dense_a && dense_b) {
      const auto* x = a.data();
      const auto* y = b.data();
      for (std::size_t i = 0; i < out.size(); ++i) out.data()[i] = f(x[i], y[i]);
      return out;
    }
    const strides_type sa = broadcast_strides(a.shape(), a.strides(), s);
    const strides_type sb = broadcast_strides(b.shape(), b.strides(), s);
    std::vector<std::ptrdiff_t> ob;
    ob.reserve(out.size());
    for_each_offset(s, sb, b.data_offset(), [&](std::ptrdiff_t o) { ob.push_back(o); });
    const auto* x = a.data();
    const auto* y = b.data();
    std::size_t k = 0;
    for_each_offset(s, sa, a.data_offset(), [&](std::ptrdiff_t o) {
      out.data()[k] = f(x[o], y[ob[k]]);
      ++k;
    });
    return out;
  }
}

template <class A, class B>
inline constexpr bool binary_ok_v =
    (is_xexpr_v<A> && (is_xexpr_v<B> || is_scalar_v<B>)) || (is_scalar_v<A> && is_xexpr_v<B>);

}  // namespace detail

// ---------------------------------------------------------------- operators
#define XT_SUBSET_BINARY(OP)                                                              \
  template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>      \
  auto operator OP(const A& a, const B& b) {                                              \
    return detail::map2([](const auto& x, const auto& y) { return x OP y; }, a, b);       \
  }
XT_SUBSET_BINARY(+)
XT_SUBSET_BINARY(-)
XT_SUBSET_BINARY(*)
XT_SUBSET_BINARY(/)
XT_SUBSET_BINARY(<)
XT_SUBSET_BINARY(>)
XT_SUBSET_BINARY(<=)
XT_SUBSET_BINARY(>=)
XT_SUBSET_BINARY(&&)
XT_SUBSET_BINARY(||)
#undef XT_SUBSET_BINARY

template <class A, std::enable_if_t<is_xexpr_v<A>, int> = 0>
auto operator-(const A& a) {
  return detail::map1([](const auto& x) { return -x; }, a);
}
template <class A, std::enable_if_t<is_xexpr_v<A>, int> = 0>
auto operator+(const A& a) {
  return detail::map1([](const auto& x) { return +x; }, a);
}
template <class A, std::enable_if_t<is_xexpr_v<A>, int> = 0>
auto operator!(const A& a) {
  return detail::map1([](const auto& x) { return !x; }, a);
}

// == and != compare whole expressions (shape and every element), as in xtensor.
template <class A, class B, std::enable_if_t<is_xexpr_v<A> && is_xexpr_v<B>, int> = 0>
bool operator==(const A& a, const B& b) {
  if (a.shape() != b.shape()) return false;
  const auto x = eval(a);
  const auto y = eval(b);
  for (std::size_t i = 0; i < x.size(); ++i)
    if (!(x.data()[i] == y.data()[i])) return false;
  return true;
}
template <class A, class B, std::enable_if_t<is_xexpr_v<A> && is_xexpr_v<B>, int> = 0>
bool operator!=(const A& a, const B& b) {
  return !(a == b);
}

// Compound assignment on containers (broadcast to the container's shape).
#define XT_SUBSET_COMPOUND(OP, F)                                                         \
  template <class T, class E>                                                             \
  xdense<T>& operator OP(xdense<T>& c, const E& e) {                                      \
    if constexpr (is_scalar_v<E>) {                                                       \
      for (auto& v : c) v = (T)(F()(v, e));                                               \
    } else {                                                                              \
      const xarray<T> t(e);                                                               \
      std::vector<T> tmp(c.size());                                                       \
      detail::copy_broadcast(t, c.shape(), tmp.data());                                   \
      for (std::size_t i = 0; i < c.size(); ++i) c.data()[i] = (T)(F()(c.data()[i], tmp[i])); \
    }                                                                                     \
    return c;                                                                             \
  }
XT_SUBSET_COMPOUND(+=, std::plus<>)
XT_SUBSET_COMPOUND(-=, std::minus<>)
XT_SUBSET_COMPOUND(*=, std::multiplies<>)
XT_SUBSET_COMPOUND(/=, std::divides<>)
#undef XT_SUBSET_COMPOUND

// ---------------------------------------------------------------- math
#define XT_SUBSET_UNARY(NAME, EXPR)                                                       \
  template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>                            \
  auto NAME(const E& e) {                                                                 \
    return detail::map1([](const auto& x) { using std::NAME; return EXPR; }, e);          \
  }
XT_SUBSET_UNARY(sin, sin(x))
XT_SUBSET_UNARY(cos, cos(x))
XT_SUBSET_UNARY(tan, tan(x))
XT_SUBSET_UNARY(exp, exp(x))
XT_SUBSET_UNARY(log, log(x))
XT_SUBSET_UNARY(sqrt, sqrt(x))
XT_SUBSET_UNARY(abs, abs(x))
XT_SUBSET_UNARY(fabs, fabs(x))
XT_SUBSET_UNARY(floor, floor(x))
XT_SUBSET_UNARY(ceil, ceil(x))
XT_SUBSET_UNARY(round, round(x))
XT_SUBSET_UNARY(atan, atan(x))
XT_SUBSET_UNARY(asin, asin(x))
XT_SUBSET_UNARY(acos, acos(x))
XT_SUBSET_UNARY(real, real(x))
XT_SUBSET_UNARY(imag, imag(x))
XT_SUBSET_UNARY(conj, conj(x))
XT_SUBSET_UNARY(norm, norm(x))
XT_SUBSET_UNARY(arg, arg(x))
#undef XT_SUBSET_UNARY

template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>
auto pow(const A& a, const B& b) {
  return detail::map2([](const auto& x, const auto& y) { using std::pow; return pow(x, y); }, a,
                      b);
}
template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>
auto atan2(const A& a, const B& b) {
  return detail::map2([](const auto& x, const auto& y) { using std::atan2; return atan2(x, y); },
                      a, b);
}
template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>
auto maximum(const A& a, const B& b) {
  return detail::map2([](const auto& x, const auto& y) { return x > y ? x : y; }, a, b);
}
template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>
auto minimum(const A& a, const B& b) {
  return detail::map2([](const auto& x, const auto& y) { return x < y ? x : y; }, a, b);
}
template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>
auto equal(const A& a, const B& b) {
  return detail::map2([](const auto& x, const auto& y) { return x == y; }, a, b);
}
template <class A, class B, std::enable_if_t<detail::binary_ok_v<A, B>, int> = 0>
auto not_equal(const A& a, const B& b) {
  return detail::map2([](const auto& x, const auto& y) { return x != y; }, a, b);
}
template <class C, class A, class B>
auto where(const C& c, const A& a, const B& b) {
  const auto cc = eval(c);
  using R = std::common_type_t<std::conditional_t<is_scalar_v<A>, A, detail::value_t<A>>,
                               std::conditional_t<is_scalar_v<B>, B, detail::value_t<B>>>;
  auto full = [&](const auto& x) {
    if constexpr (is_scalar_v<std::decay_t<decltype(x)>>) {
      return xarray<R>(cc.shape(), (R)x);
    } else {
      xarray<R> t = xarray<R>::from_shape(cc.shape());
      detail::copy_broadcast(x, cc.shape(), t.data());
      return t;
    }
  };
  const xarray<R> ea = full(a), eb = full(b);
  xarray<R> out = xarray<R>::from_shape(cc.shape());
  for (std::size_t i = 0; i < out.size(); ++i)
    out.data()[i] = cc.data()[i] ? ea.data()[i] : eb.data()[i];
  return out;
}

// make_lambda_xfunction(f, e...): f applied element-wise.
template <class F, class E>
auto make_lambda_xfunction(F&& f, const E& e) {
  return detail::map1(f, e);
}
template <class F, class A, class B>
auto make_lambda_xfunction(F&& f, const A& a, const B& b) {
  return detail::map2(f, a, b);
}

// ---------------------------------------------------------------- reducers
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto sum(const E& e) {
  const auto x = eval(e);
  using T = detail::value_t<E>;
  T s = T(0);
  for (const auto& v : x) s += v;
  return xarray<T>(shape_type{}, s);
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto amin(const E& e) {
  const auto x = eval(e);
  if (x.size() == 0) throw std::runtime_error("xt::amin of an empty expression");
  return xarray<detail::value_t<E>>(shape_type{}, *std::min_element(x.begin(), x.end()));
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto amax(const E& e) {
  const auto x = eval(e);
  if (x.size() == 0) throw std::runtime_error("xt::amax of an empty expression");
  return xarray<detail::value_t<E>>(shape_type{}, *std::max_element(x.begin(), x.end()));
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
bool any(const E& e) {
  const auto x = eval(e);
  for (const auto& v : x)
    if (v) return true;
  return false;
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
bool all(const E& e) {
  const auto x = eval(e);
  for (const auto& v : x)
    if (!v) return false;
  return true;
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto norm_l2(const E& e) {
  const auto x = eval(e);
  using V = detail::value_t<E>;
  using R = decltype(std::abs(std::declval<V>()));
  R s = R(0);
  for (const auto& v : x) {
    const R a = std::abs(v);
    s += a * a;
  }
  return xarray<R>(shape_type{}, std::sqrt(s));
}
// Flat (row-major) index of the first minimum.
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto argmin(const E& e) {
  const auto x = eval(e);
  if (x.size() == 0) throw std::runtime_error("xt::argmin of an empty expression");
  return xarray<std::size_t>(shape_type{},
                             (std::size_t)(std::min_element(x.begin(), x.end()) - x.begin()));
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto argmax(const E& e) {
  const auto x = eval(e);
  if (x.size() == 0) throw std::runtime_error("xt::argmax of an empty expression");
  return xarray<std::size_t>(shape_type{},
                             (std::size_t)(std::max_element(x.begin(), x.end()) - x.begin()));
}
// Sorted distinct values, 1-D.
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto unique(const E& e) {
  const auto x = eval(e);
  std::vector<detail::value_t<E>> v(x.begin(), x.end());
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  xarray<detail::value_t<E>> out = xarray<detail::value_t<E>>::from_shape(shape_type{v.size()});
  std::copy(v.begin(), v.end(), out.begin());
  return out;
}
// Reversed along `axis`.
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto flip(const E& e, std::size_t axis = 0) {
  const auto x = eval(e);
  using T = detail::value_t<E>;
  strides_type st = detail::plain_strides(x);
  std::ptrdiff_t off = (std::ptrdiff_t)(x.shape()[axis] - 1) * st[axis];
  st[axis] = -st[axis];
  const xview<const T> v(x.data(), off, x.shape(), st);
  return xarray<T>(v);
}

// ---------------------------------------------------------------- builders
template <class T, class S>
xarray<T> zeros(const S& s) {
  return xarray<T>(shape_type(std::begin(s), std::end(s)), T(0));
}
template <class T>
xarray<T> zeros(std::initializer_list<std::size_t> s) {
  return xarray<T>(shape_type(s), T(0));
}
template <class T, class S>
xarray<T> ones(const S& s) {
  return xarray<T>(shape_type(std::begin(s), std::end(s)), T(1));
}
template <class T>
xarray<T> ones(std::initializer_list<std::size_t> s) {
  return xarray<T>(shape_type(s), T(1));
}
template <class T, class S>
xarray<T> empty(const S& s) {
  return xarray<T>(shape_type(std::begin(s), std::end(s)));
}
template <class T>
xarray<T> empty(std::initializer_list<std::size_t> s) {
  return xarray<T>(shape_type(s));
}
// *_like: a container of the operand's own type (xarray for a view).
namespace detail {
template <class E>
struct like_type {
  using type = xarray<value_t<E>>;
};
template <class T, std::size_t N>
struct like_type<xtensor<T, N>> {
  using type = xtensor<T, N>;
};
template <class T, std::size_t... I>
struct like_type<xtensor_fixed<T, xshape<I...>>> {
  using type = xtensor_fixed<T, xshape<I...>>;
};
template <class E>
auto make_like(const E& e, const value_t<E>* fill) {
  using C = typename like_type<std::decay_t<E>>::type;
  xarray<value_t<E>> a = fill ? xarray<value_t<E>>(e.shape(), *fill)
                              : xarray<value_t<E>>(e.shape());
  if constexpr (std::is_same_v<C, xarray<value_t<E>>>) return a;
  else return C(std::move(a));
}
}  // namespace detail
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto zeros_like(const E& e) {
  const detail::value_t<E> v(0);
  return detail::make_like(e, &v);
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto ones_like(const E& e) {
  const detail::value_t<E> v(1);
  return detail::make_like(e, &v);
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto empty_like(const E& e) {
  return detail::make_like(e, static_cast<const detail::value_t<E>*>(nullptr));
}
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
auto full_like(const E& e, detail::value_t<E> v) {
  return detail::make_like(e, &v);
}

// linspace: num points from start to stop (stop included when endpoint),
// value i = start + i * step.
template <class T>
xarray<T> linspace(T start, T stop, std::size_t num = 50, bool endpoint = true) {
  xarray<T> out = xarray<T>::from_shape(shape_type{num});
  const T step = (stop - start) / T(num - (endpoint ? 1 : 0));
  for (std::size_t i = 0; i < num; ++i) out.data()[i] = start + step * T(i);
  if (endpoint && num > 1) out.data()[num - 1] = stop;
  return out;
}
// arange(start, stop, step): start + i * step while below stop (above, for a
// negative step).  The value type is the explicit template argument, else the
// common type of the arguments.
namespace detail {
template <class T, class... A>
using arange_t = std::conditional_t<std::is_void_v<T>, std::common_type_t<A...>, T>;
}
template <class T = void, class A, class B, class C>
xarray<detail::arange_t<T, A, B, C>> arange(A start, B stop, C step) {
  using R = detail::arange_t<T, A, B, C>;
  const R a = (R)start, b = (R)stop, s = (R)step;
  const std::size_t n =
      s > R(0) ? (b > a ? (std::size_t)std::ceil((double)(b - a) / (double)s) : 0)
               : (a > b ? (std::size_t)std::ceil((double)(a - b) / (double)(-s)) : 0);
  xarray<R> out = xarray<R>::from_shape(shape_type{n});
  for (std::size_t i = 0; i < n; ++i) out.data()[i] = (R)(a + (R)i * s);
  return out;
}
template <class T = void, class A, class B>
xarray<detail::arange_t<T, A, B>> arange(A start, B stop) {
  return arange<detail::arange_t<T, A, B>>(start, stop, 1);
}
template <class T = void, class B>
xarray<detail::arange_t<T, B>> arange(B stop) {
  return arange<detail::arange_t<T, B>>(0, stop, 1);
}

// xtuple: the operands of concatenate / stack.
template <class... E>
auto xtuple(E&&... e) {
  return std::make_tuple(eval(std::forward<E>(e))...);
}

template <class... E>
auto concatenate(const std::tuple<E...>& t, std::size_t axis = 0) {
  using T = std::common_type_t<detail::value_t<E>...>;
  std::vector<xarray<T>> parts;
  std::apply([&](const auto&... a) { (parts.push_back(xarray<T>(a)), ...); }, t);
  shape_type s = parts.front().shape();
  std::size_t total = 0;
  for (const auto& p : parts) total += p.shape()[axis];
  s[axis] = total;
  xarray<T> out = xarray<T>::from_shape(s);
  std::size_t at = 0;
  const strides_type st = detail::plain_strides(out);
  for (const auto& p : parts) {
    shape_type ds = out.shape();
    ds[axis] = p.shape()[axis];
    xview<T>(out.data(), (std::ptrdiff_t)at * st[axis], ds, st) = p;
    at += ds[axis];
  }
  return out;
}

template <class... E>
auto stack(const std::tuple<E...>& t, std::size_t axis = 0) {
  using T = std::common_type_t<detail::value_t<E>...>;
  std::vector<xarray<T>> parts;
  std::apply([&](const auto&... a) { (parts.push_back(xarray<T>(a)), ...); }, t);
  shape_type s = parts.front().shape();
  s.insert(s.begin() + (std::ptrdiff_t)axis, parts.size());
  xarray<T> out = xarray<T>::from_shape(s);
  const strides_type st = detail::plain_strides(out);
  shape_type ps = parts.front().shape();
  strides_type pst = st;
  pst.erase(pst.begin() + (std::ptrdiff_t)axis);
  for (std::size_t q = 0; q < parts.size(); ++q)
    xview<T>(out.data(), (std::ptrdiff_t)q * st[axis], ps, pst) = parts[q];
  return out;
}

// meshgrid with 'ij' indexing: output q varies along axis q.
template <class... E>
auto meshgrid(const E&... e) {
  constexpr std::size_t n = sizeof...(E);
  using T = std::common_type_t<detail::value_t<E>...>;
  std::array<xarray<T>, n> in{xarray<T>(e)...};
  shape_type s(n);
  for (std::size_t q = 0; q < n; ++q) s[q] = in[q].size();
  auto build = [&](std::size_t q) {
    xarray<T> out = xarray<T>::from_shape(s);
    std::size_t k = 0;
    strides_type bs(n, 0);
    bs[q] = 1;
    detail::for_each_offset(s, bs, 0, [&](std::ptrdiff_t o) { out.data()[k++] = in[q].data()[o]; });
    return out;
  };
  return [&]<std::size_t... I>(std::index_sequence<I...>) {
    return std::make_tuple(build(I)...);
  }(std::make_index_sequence<n>{});
}

// adapt: a 1-D array holding a copy of a sequence's values.
template <class C>
auto adapt(const C& c) {
  using T = std::decay_t<decltype(*std::begin(c))>;
  xarray<T> out = xarray<T>::from_shape(shape_type{(std::size_t)std::distance(std::begin(c), std::end(c))});
  std::copy(std::begin(c), std::end(c), out.begin());
  return out;
}
template <class T, class S>
auto adapt(T* p, std::size_t n, int /*ownership*/, const S& shape) {
  xarray<T> out = xarray<T>::from_shape(shape_type(std::begin(shape), std::end(shape)));
  std::copy(p, p + n, out.begin());
  return out;
}

// ---------------------------------------------------------------- printing
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
std::ostream& operator<<(std::ostream& os, const E& e) {
  const auto x = eval(e);
  os << "{";
  for (std::size_t i = 0; i < x.size(); ++i) os << (i ? ", " : "") << x.data()[i];
  os << "}";
  return os;
}

// ---------------------------------------------------------------- .npy
namespace detail {
template <class T>
std::string npy_descr() {
  if constexpr (std::is_same_v<T, double>) return "<f8";
  else if constexpr (std::is_same_v<T, float>) return "<f4";
  else if constexpr (std::is_same_v<T, std::complex<double>>) return "<c16";
  else if constexpr (std::is_same_v<T, std::complex<float>>) return "<c8";
  else if constexpr (std::is_same_v<T, bool>) return "|b1";
  else if constexpr (std::is_integral_v<T> && std::is_signed_v<T>)
    return "<i" + std::to_string(sizeof(T));
  else if constexpr (std::is_integral_v<T>) return "<u" + std::to_string(sizeof(T));
  else static_assert(sizeof(T) == 0, "xt::dump_npy: unsupported element type");
}
}  // namespace detail

// Writes e to `path` in NumPy's .npy format, version 1.0, C order.
template <class E, std::enable_if_t<is_xexpr_v<E>, int> = 0>
void dump_npy(const std::string& path, const E& e) {
  using T = detail::value_t<E>;
  const xarray<T> x(e);
  std::ostringstream dict;
  dict << "{'descr': '" << detail::npy_descr<T>() << "', 'fortran_order': False, 'shape': (";
  for (std::size_t d = 0; d < x.shape().size(); ++d) {
    dict << x.shape()[d];
    if (x.shape().size() == 1 || d + 1 < x.shape().size()) dict << ",";
    if (d + 1 < x.shape().size()) dict << " ";
  }
  dict << "), }";
  std::string h = dict.str();
  const std::size_t pre = 10;  // magic (6) + version (2) + header length (2)
  std::size_t total = pre + h.size() + 1;
  const std::size_t padded = (total + 63) / 64 * 64;
  h.append(padded - total, ' ');
  h.push_back('\n');
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("xt::dump_npy: cannot open " + path);
  const char magic[8] = {'\x93', 'N', 'U', 'M', 'P', 'Y', 1, 0};
  f.write(magic, 8);
  const uint16_t hl = (uint16_t)h.size();
  const char hb[2] = {(char)(hl & 0xff), (char)(hl >> 8)};
  f.write(hb, 2);
  f.write(h.data(), (std::streamsize)h.size());
  f.write(reinterpret_cast<const char*>(x.data()), (std::streamsize)(x.size() * sizeof(T)));
}

}  // namespace xt

// Programs written for xtensor name the open-range placeholder unqualified.
using xt::placeholders::_;
