/* empty stand-in for <random/beta.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
