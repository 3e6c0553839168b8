/* empty stand-in for <random/chisquare.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
