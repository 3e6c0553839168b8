/* Declaration-only stand-in for <fftw3-mpi.h>: the plan handle type the reference's headers
 * declare extern variables of; no FFTW function is called (test infrastructure only). */
#pragma once
#include <cstddef>
typedef struct tg_stub_fftw_plan_s* fftw_plan;
