/*
 * flups_mpi.h -- the MPI communicator type used in the FLUPS C API.
 *
 * The reference's API takes an MPI_Comm (src/flups.h:210, :329).  This
 * library runs on one device with a size-1 communicator: compiled with
 * -DFLUPS_HAVE_MPI the real <mpi.h> is used (and the communicator must have
 * size 1); otherwise a pointer-sized stand-in is declared so that callers
 * without MPI can pass MPI_COMM_WORLD.
 */
#ifndef FLUPS_MPI_H
#define FLUPS_MPI_H
#ifdef FLUPS_HAVE_MPI
#include <mpi.h>
#else
#include <stdint.h>
typedef intptr_t MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#endif
#endif
#endif
