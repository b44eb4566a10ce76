/* Single-rank stand-in for MPI-IO, pulled in by the HDF5 headers; the oracle
 * never performs parallel I/O. */
#ifndef PHX_ORACLE_MPIO_SHIM_H
#define PHX_ORACLE_MPIO_SHIM_H
#include "mpi.h"
#endif
