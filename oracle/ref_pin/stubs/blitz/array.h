/* Declaration-only stand-in for <blitz/array.h>: the names the reference's inline wavenumber
 * headers mention (Array in signatures of functions the pin harness never calls, and the scalar
 * pow2 they do call), so that those headers compile without blitz++ (test infrastructure only). */
#pragma once
#include <cmath>
#include <complex>
#include <string>
using namespace std;
namespace blitz {
template <typename T, int R>
class Array {
 public:
  T& operator()(int, int, int);
  T operator()(int, int, int) const;
};
template <typename T, int R>
class TinyVector {};
inline double pow2(double x) { return x * x; }
}  // namespace blitz
