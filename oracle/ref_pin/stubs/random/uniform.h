/* Declaration-only stand-in for blitz <random/uniform.h>: the generator type the reference
 * declares an extern variable of; never used by the pin harness (test infrastructure only). */
#pragma once
namespace ranlib {
template <typename T>
class Uniform {};
}  // namespace ranlib
