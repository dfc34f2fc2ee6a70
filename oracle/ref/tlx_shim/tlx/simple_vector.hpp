// Project-written stand-in: a fixed-size array with the interface the
// reference's Point storage uses (sized construction, resize, size, element
// access, iterators); the initialisation modes are accepted and ignored.
#pragma once
#include <cstddef>
#include <vector>

namespace tlx {
enum class SimpleVectorMode { Normal, NoInitButDestroy, NoInitNoDestroy };

template <typename T, SimpleVectorMode Mode = SimpleVectorMode::Normal>
class SimpleVector {
  public:
    using iterator = T *;
    using const_iterator = const T *;
    SimpleVector() = default;
    explicit SimpleVector(std::size_t n) : v_(n) {}
    SimpleVector(SimpleVector &&) noexcept = default;
    SimpleVector &operator=(SimpleVector &&) noexcept = default;
    std::size_t size() const noexcept { return v_.size(); }
    void resize(std::size_t n) { v_.resize(n); }
    T &operator[](std::size_t i) noexcept { return v_[i]; }
    const T &operator[](std::size_t i) const noexcept { return v_[i]; }
    T *data() noexcept { return v_.data(); }
    const T *data() const noexcept { return v_.data(); }
    iterator begin() noexcept { return v_.data(); }
    iterator end() noexcept { return v_.data() + v_.size(); }
    const_iterator begin() const noexcept { return v_.data(); }
    const_iterator end() const noexcept { return v_.data() + v_.size(); }

  private:
    std::vector<T> v_;
};
} // namespace tlx
