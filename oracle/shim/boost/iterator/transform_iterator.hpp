// Oracle-build stand-in: declarations only (see zip_iterator.hpp).
#pragma once
namespace boost {
template <class F, class It> class transform_iterator;
template <class F, class It> transform_iterator<F, It> make_transform_iterator(It it, F f);
}  // namespace boost
