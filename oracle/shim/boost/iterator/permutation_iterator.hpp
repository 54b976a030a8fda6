// Oracle-build stand-in: declarations only (see zip_iterator.hpp).
#pragma once
namespace boost {
template <class Elements, class Index> class permutation_iterator;
template <class Elements, class Index>
permutation_iterator<Elements, Index> make_permutation_iterator(Elements e, Index i);
}  // namespace boost
