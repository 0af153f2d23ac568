// Test stand-in for green::ndarray::ndarray (the array type of green-mbpt's ztensor<N>): row-major
// storage, shape(), data(), copy(), set_zero() and views of the leading indices, the members the
// B200 plug-in uses.  Test infrastructure only.
#pragma once
#include <array>
#include <complex>
#include <cstddef>
#include <memory>
#include <vector>

namespace green::ndarray {

template <typename T, size_t D>
class ndarray {
 public:
  ndarray() = default;
  explicit ndarray(const std::array<size_t, D>& shape)
      : shape_(shape), own_(std::make_shared<std::vector<T>>(count(shape))), ptr_(own_->data()) {}
  template <typename... I, typename = std::enable_if_t<sizeof...(I) + 1 == D>>
  explicit ndarray(size_t a, I... rest) : ndarray(std::array<size_t, D>{a, size_t(rest)...}) {}
  ndarray(T* ptr, const std::array<size_t, D>& shape, std::shared_ptr<std::vector<T>> own = nullptr)
      : shape_(shape), own_(std::move(own)), ptr_(ptr) {}

  const std::array<size_t, D>& shape() const { return shape_; }
  size_t size() const { return count(shape_); }
  T* data() { return ptr_; }
  const T* data() const { return ptr_; }
  void set_zero() { std::fill(ptr_, ptr_ + size(), T(0)); }
  ndarray copy() const {
    ndarray c(shape_);
    std::copy(ptr_, ptr_ + size(), c.data());
    return c;
  }
  // view of the sub-array at the leading indices
  template <typename... I>
  ndarray<T, D - sizeof...(I)> operator()(I... idx) const {
    constexpr size_t K = sizeof...(I);
    const size_t ix[K] = {size_t(idx)...};
    size_t off = 0;
    for (size_t d = 0; d < K; ++d) off = off * shape_[d] + ix[d];
    std::array<size_t, D - K> sub{};
    size_t inner = 1;
    for (size_t d = K; d < D; ++d) {
      sub[d - K] = shape_[d];
      inner *= shape_[d];
    }
    return ndarray<T, D - K>(ptr_ + off * inner, sub, own_);
  }

 private:
  static size_t count(const std::array<size_t, D>& s) {
    size_t n = 1;
    for (size_t x : s) n *= x;
    return n;
  }
  std::array<size_t, D> shape_{};
  std::shared_ptr<std::vector<T>> own_;
  T* ptr_ = nullptr;
};

}  // namespace green::ndarray
