/* Declaration-only stand-in for <mpi.h>: enough for the reference's inline wavenumber headers to
 * parse in a one-process build that calls no MPI function (test infrastructure only). */
#pragma once
typedef struct { int source, tag, error; } MPI_Status;
