// template_array.hpp -- TArray<T>, the structure-of-arrays container of the
// host interface.
//
// Interface of the reference's TArray (src/template_array.hpp:9-90): up to
// four dimensions indexed (n, k, j, i) with i fastest, zero-initialised
// storage, deep copy, move, Swap.  Storage is a std::vector here.
#pragma once

#include <cstddef>
#include <utility>
#include <vector>

namespace Gaukuk {

template <class T>
class TArray {
public:
    enum class ArrayStatus { empty, allocated };

    TArray() = default;
    explicit TArray(int n1) { Allocate(1, 1, 1, n1); }
    TArray(int n2, int n1) { Allocate(1, 1, n2, n1); }
    TArray(int n3, int n2, int n1) { Allocate(1, n3, n2, n1); }
    TArray(int n4, int n3, int n2, int n1) { Allocate(n4, n3, n2, n1); }

    void NewArray(int n1) { Allocate(1, 1, 1, n1); }
    void NewArray(int n2, int n1) { Allocate(1, 1, n2, n1); }
    void NewArray(int n3, int n2, int n1) { Allocate(1, n3, n2, n1); }
    void NewArray(int n4, int n3, int n2, int n1) { Allocate(n4, n3, n2, n1); }

    size_t GetSize() const { return v_.size(); }
    size_t GetSizeInBytes() const { return v_.size() * sizeof(T); }
    int GetN1() const { return n1_; }
    int GetN2() const { return n2_; }
    int GetN3() const { return n3_; }
    int GetN4() const { return n4_; }

    T& operator()(int i) { return v_[i]; }
    T operator()(int i) const { return v_[i]; }
    T& operator()(int n, int i) { return v_[i + (size_t)n1_ * n]; }
    T operator()(int n, int i) const { return v_[i + (size_t)n1_ * n]; }
    T& operator()(int n, int j, int i) { return v_[i + (size_t)n1_ * (j + (size_t)n2_ * n)]; }
    T operator()(int n, int j, int i) const { return v_[i + (size_t)n1_ * (j + (size_t)n2_ * n)]; }
    T& operator()(int n, int k, int j, int i) {
        return v_[i + (size_t)n1_ * (j + (size_t)n2_ * (k + (size_t)n3_ * n))];
    }
    T operator()(int n, int k, int j, int i) const {
        return v_[i + (size_t)n1_ * (j + (size_t)n2_ * (k + (size_t)n3_ * n))];
    }

    T* data() noexcept { return v_.empty() ? nullptr : v_.data(); }
    const T* data() const noexcept { return v_.empty() ? nullptr : v_.data(); }

    void Swap(TArray& o) noexcept {
        std::swap(n1_, o.n1_);
        std::swap(n2_, o.n2_);
        std::swap(n3_, o.n3_);
        std::swap(n4_, o.n4_);
        v_.swap(o.v_);
    }
    void DeleteArray() noexcept {
        std::vector<T>().swap(v_);
        n1_ = n2_ = n3_ = n4_ = 0;
    }
    ArrayStatus Status() const { return v_.empty() ? ArrayStatus::empty : ArrayStatus::allocated; }

private:
    void Allocate(int n4, int n3, int n2, int n1) {
        n1_ = n1; n2_ = n2; n3_ = n3; n4_ = n4;
        std::vector<T>((size_t)n1 * n2 * n3 * n4, T()).swap(v_);
    }
    std::vector<T> v_;
    int n1_ = 0, n2_ = 0, n3_ = 0, n4_ = 0;
};

}  // namespace Gaukuk
