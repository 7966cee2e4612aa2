// Minimal stand-ins for the handful of Boost names the Cyclops engine headers
// mention.  Test infrastructure only: it lets the reference engine compile
// from its own sources for use as the CPU oracle.  Only what the engine
// actually instantiates (tuple/get) has working semantics; the iterator
// adaptors exist so that uninstantiated templates parse.
#ifndef CYC_BOOST_SHIM_HPP
#define CYC_BOOST_SHIM_HPP
#include <tuple>
#include <iterator>
#include <cstddef>
#include <utility>

namespace boost {
namespace tuples {
template <class... T> using tuple = std::tuple<T...>;
}
template <class... T> using tuple = std::tuple<T...>;
using std::get;
using std::make_tuple;

template <class T>
class counting_iterator {
public:
    typedef std::random_access_iterator_tag iterator_category;
    typedef T value_type;
    typedef std::ptrdiff_t difference_type;
    typedef const T* pointer;
    typedef const T& reference;
    counting_iterator() : v() {}
    explicit counting_iterator(T x) : v(x) {}
    const T& operator*() const { return v; }
    counting_iterator& operator++() { ++v; return *this; }
    counting_iterator operator++(int) { counting_iterator r(*this); ++v; return r; }
    counting_iterator& operator--() { --v; return *this; }
    counting_iterator& operator+=(difference_type n) { v += n; return *this; }
    counting_iterator operator+(difference_type n) const { return counting_iterator(v + n); }
    difference_type operator-(const counting_iterator& o) const { return v - o.v; }
    bool operator==(const counting_iterator& o) const { return v == o.v; }
    bool operator!=(const counting_iterator& o) const { return v != o.v; }
    bool operator<(const counting_iterator& o) const { return v < o.v; }
private:
    T v;
};
template <class T> counting_iterator<T> make_counting_iterator(T x) { return counting_iterator<T>(x); }

template <class Tuple> class zip_iterator {
public:
    zip_iterator() {}
    explicit zip_iterator(const Tuple& t) : t(t) {}
    Tuple t;
};
template <class Tuple> zip_iterator<Tuple> make_zip_iterator(const Tuple& t) { return zip_iterator<Tuple>(t); }

template <class It> class iterator_range {
public:
    iterator_range(It b, It e) : b(b), e(e) {}
    It begin() const { return b; }
    It end() const { return e; }
private:
    It b, e;
};

template <class Elem, class Index> class permutation_iterator {
public:
    permutation_iterator() {}
    permutation_iterator(Elem e, Index i) : e(e), i(i) {}
    Elem e; Index i;
};
template <class Elem, class Index>
permutation_iterator<Elem, Index> make_permutation_iterator(Elem e, Index i) {
    return permutation_iterator<Elem, Index>(e, i);
}

template <class F, class It> class transform_iterator {
public:
    transform_iterator() {}
    transform_iterator(It it, F f) : it(it), f(f) {}
    It it; F f;
};
template <class F, class It> transform_iterator<F, It> make_transform_iterator(It it, F f) {
    return transform_iterator<F, It>(it, f);
}
} // namespace boost
#endif
