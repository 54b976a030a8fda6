// Oracle-build stand-in for boost::counting_iterator: a random-access iterator
// over consecutive integers, enough for the reference's serial loop helpers.
#pragma once
#include <cstddef>
#include <iterator>
namespace boost {
template <class Int>
class counting_iterator {
public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type = Int;
    using difference_type = std::ptrdiff_t;
    using pointer = const Int*;
    using reference = Int;
    counting_iterator() : v_() {}
    explicit counting_iterator(Int v) : v_(v) {}
    Int operator*() const { return v_; }
    Int operator[](difference_type n) const { return static_cast<Int>(v_ + n); }
    counting_iterator& operator++() { ++v_; return *this; }
    counting_iterator operator++(int) { counting_iterator t(*this); ++v_; return t; }
    counting_iterator& operator--() { --v_; return *this; }
    counting_iterator& operator+=(difference_type n) { v_ = static_cast<Int>(v_ + n); return *this; }
    counting_iterator& operator-=(difference_type n) { v_ = static_cast<Int>(v_ - n); return *this; }
    friend counting_iterator operator+(counting_iterator a, difference_type n) { return a += n; }
    friend counting_iterator operator+(difference_type n, counting_iterator a) { return a += n; }
    friend counting_iterator operator-(counting_iterator a, difference_type n) { return a -= n; }
    friend difference_type operator-(const counting_iterator& a, const counting_iterator& b) {
        return static_cast<difference_type>(a.v_) - static_cast<difference_type>(b.v_);
    }
    friend bool operator==(const counting_iterator& a, const counting_iterator& b) { return a.v_ == b.v_; }
    friend bool operator!=(const counting_iterator& a, const counting_iterator& b) { return a.v_ != b.v_; }
    friend bool operator<(const counting_iterator& a, const counting_iterator& b) { return a.v_ < b.v_; }
private:
    Int v_;
};
template <class Int>
counting_iterator<Int> make_counting_iterator(Int v) { return counting_iterator<Int>(v); }
}  // namespace boost
