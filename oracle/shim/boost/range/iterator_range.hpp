// Oracle-build stand-in for boost::iterator_range: a [begin, end) pair. The
// reference's range helpers (engine/Ranges.h) return it from non-template
// functions, so the type must be complete; none of them is called on the
// coordinate-descent path.
#pragma once
namespace boost {
template <class It>
class iterator_range {
public:
    iterator_range(It b, It e) : b_(b), e_(e) {}
    It begin() const { return b_; }
    It end() const { return e_; }
private:
    It b_, e_;
};
}  // namespace boost
