// Rcpp.h -- a stand-in for the few Rcpp types that the reference's src/predict.cpp uses, so that file compiles
// unmodified here as a parity oracle (R and Rcpp are not installed).  TEST INFRASTRUCTURE ONLY: built by
// oracle/Makefile into oracle/_ref/libpredref.so together with oracle/ref_predict_shim.cpp.
//
// Covered: Rcpp::List (index by position or name, List::create with Rcpp::Named), Rcpp::NumericVector, Rcpp::as for
// int / std::vector<double> / NumericVector, Rcpp::stop (printf-style message, thrown as std::runtime_error), and R's
// INTEGER() / REAL() accessors on list elements.  A list element holds either an integer or a double vector.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace Rcpp {

struct Value {
  std::vector<int> i;
  std::vector<double> d;
  bool is_int = false;
  Value() {}
  Value(int x) : i{x}, is_int(true) {}
  Value(const std::vector<int>& v) : i(v), is_int(true) {}
  Value(const std::vector<double>& v) : d(v) {}
};

class NumericVector {
 public:
  NumericVector() {}
  explicit NumericVector(int n) : v(static_cast<size_t>(n), 0.0) {}
  explicit NumericVector(const std::vector<double>& x) : v(x) {}
  double* begin() { return v.data(); }
  int size() const { return static_cast<int>(v.size()); }
  std::vector<double> v;
};

struct NamedValue {
  std::string name;
  Value value;
};

struct Named {
  std::string name;
  explicit Named(const char* n) : name(n) {}
  template <class T>
  NamedValue operator=(const T& x) const { return NamedValue{name, Value(x)}; }
};

class List {
 public:
  std::vector<NamedValue> items;
  int size() const { return static_cast<int>(items.size()); }
  Value& operator[](int k) { return items.at(static_cast<size_t>(k)).value; }
  Value& operator[](const char* name) {
    for (auto& it : items)
      if (it.name == name) return it.value;
    throw std::runtime_error(std::string("no list element ") + name);
  }
  template <class... A>
  static List create(A&&... a) {
    List l;
    (l.items.push_back(std::forward<A>(a)), ...);
    return l;
  }
};

template <class T>
T as(const Value& v);
template <>
inline int as<int>(const Value& v) { return v.is_int ? v.i.at(0) : static_cast<int>(v.d.at(0)); }
template <>
inline std::vector<double> as<std::vector<double>>(const Value& v) { return v.d; }
template <>
inline NumericVector as<NumericVector>(const Value& v) { return NumericVector(v.d); }

[[noreturn]] inline void stop(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw std::runtime_error(buf);
}

}  // namespace Rcpp

inline int* INTEGER(Rcpp::Value& v) { return v.i.data(); }
inline double* REAL(Rcpp::Value& v) { return v.d.data(); }
