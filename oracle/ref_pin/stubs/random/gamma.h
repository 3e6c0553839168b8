/* empty stand-in for <random/gamma.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
