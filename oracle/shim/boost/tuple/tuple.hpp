// Oracle-build stand-in: the reference names boost tuples only as type aliases
// in its iterator traits; std::tuple provides everything that is instantiated.
#pragma once
#include <tuple>
namespace boost {
namespace tuples {
template <class... T> using tuple = std::tuple<T...>;
}  // namespace tuples
template <class... T> using tuple = std::tuple<T...>;
using std::get;
using std::make_tuple;
}  // namespace boost
