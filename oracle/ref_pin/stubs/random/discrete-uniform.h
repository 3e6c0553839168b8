/* empty stand-in for <random/discrete-uniform.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
