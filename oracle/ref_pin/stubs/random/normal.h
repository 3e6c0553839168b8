/* empty stand-in for <random/normal.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
