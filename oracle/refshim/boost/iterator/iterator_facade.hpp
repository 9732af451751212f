// Project-written minimal stand-in for <boost/iterator/iterator_facade.hpp>.
//
// Test infrastructure only: it exists so that the reference's own
// seqcsr4mlem / openmpcsr4mlem (the parity oracle) compile from their
// unmodified sources without boost installed.  The reference uses boost only
// for the CRTP iterator facade of Csr4Matrix::node_iter
// (helper_files_common/csr4matrix.hpp:84-130), which needs the private
// primitives dereference/equal/increment/decrement/advance/distance_to to be
// reachable through iterator_core_access and turned into the usual iterator
// operators.
//
// The reference instantiates the facade twice for the same Derived type (once
// as the base class, once as the `base_type` typedef with a different
// category tag), so every operator here is a member function: friend
// functions defined in the template would be defined twice.
#pragma once

#include <cstddef>
#include <iterator>
#include <type_traits>

namespace boost {

struct forward_traversal_tag {};
struct bidirectional_traversal_tag {};
struct random_access_traversal_tag {};

class iterator_core_access {
public:
    template <class It> static typename It::reference get(const It& it) { return it.dereference(); }
    template <class It> static void next(It& it) { it.increment(); }
    template <class It> static void prev(It& it) { it.decrement(); }
    template <class It, class D> static void jump(It& it, D n) { it.advance(n); }
    template <class It> static bool same(const It& a, const It& b) { return a.equal(b); }
    template <class It> static typename It::difference_type gap(const It& from, const It& to) {
        return from.distance_to(to);
    }
};

template <class Derived, class Value, class CategoryOrTraversal,
          class Reference = Value&, class Difference = std::ptrdiff_t>
class iterator_facade {
public:
    typedef std::random_access_iterator_tag iterator_category;
    typedef typename std::remove_const<Value>::type value_type;
    typedef Reference reference;
    typedef Value* pointer;
    typedef Difference difference_type;

    reference operator*() const { return iterator_core_access::get(self()); }
    pointer operator->() const { return &iterator_core_access::get(self()); }
    reference operator[](difference_type n) const { Derived t(self()); t += n; return *t; }

    Derived& operator++() { iterator_core_access::next(self()); return self(); }
    Derived operator++(int) { Derived t(self()); iterator_core_access::next(self()); return t; }
    Derived& operator--() { iterator_core_access::prev(self()); return self(); }
    Derived operator--(int) { Derived t(self()); iterator_core_access::prev(self()); return t; }
    Derived& operator+=(difference_type n) { iterator_core_access::jump(self(), n); return self(); }
    Derived& operator-=(difference_type n) { iterator_core_access::jump(self(), -n); return self(); }
    Derived operator+(difference_type n) const { Derived t(self()); t += n; return t; }
    Derived operator-(difference_type n) const { Derived t(self()); t -= n; return t; }
    difference_type operator-(const Derived& rhs) const { return iterator_core_access::gap(rhs, self()); }

    bool operator==(const Derived& rhs) const { return iterator_core_access::same(self(), rhs); }
    bool operator!=(const Derived& rhs) const { return !iterator_core_access::same(self(), rhs); }
    bool operator<(const Derived& rhs) const { return iterator_core_access::gap(self(), rhs) > 0; }
    bool operator>(const Derived& rhs) const { return iterator_core_access::gap(self(), rhs) < 0; }
    bool operator<=(const Derived& rhs) const { return iterator_core_access::gap(self(), rhs) >= 0; }
    bool operator>=(const Derived& rhs) const { return iterator_core_access::gap(self(), rhs) <= 0; }

private:
    Derived& self() { return *static_cast<Derived*>(this); }
    const Derived& self() const { return *static_cast<const Derived*>(this); }
};

}  // namespace boost
