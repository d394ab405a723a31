// Stand-in for boost::assign's `v += a, b, c;` list insertion on std::vector.
#pragma once
#include <vector>
template <class T> struct cfdv_vec_inserter {
  std::vector<T>& v;
  cfdv_vec_inserter& operator,(const T& x) { v.push_back(x); return *this; }
};
template <class T, class U> cfdv_vec_inserter<T> operator+=(std::vector<T>& v, const U& x) {
  v.push_back(x);
  return cfdv_vec_inserter<T>{v};
}
namespace boost { namespace assign { using ::operator+=; } }
