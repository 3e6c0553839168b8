/* empty stand-in for <random/F.h> (blitz random; unused by the pin harness) */
#pragma once
namespace ranlib {}
