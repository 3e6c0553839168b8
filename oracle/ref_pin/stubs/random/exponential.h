/* empty stand-in for <random/exponential.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
