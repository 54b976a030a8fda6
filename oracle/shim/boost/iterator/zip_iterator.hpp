// Oracle-build stand-in: declarations only. The reference's zip-iterator code
// (engine/Ranges.h) is never instantiated on the coordinate-descent path.
#pragma once
#include <boost/tuple/tuple.hpp>
namespace boost {
template <class Tuple> class zip_iterator;
template <class Tuple> zip_iterator<Tuple> make_zip_iterator(Tuple t);
}  // namespace boost
