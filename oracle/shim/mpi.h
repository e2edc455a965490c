/* Empty stand-in for <mpi.h>.  Test infrastructure only.
 *
 * The reference's CPU/nbody_system.cpp:2 includes <mpi.h> but uses no MPI
 * symbol, and the three reference files the oracle compiles
 * (nbody_system.cpp, force_calculation.cpp, omp_solver.cpp) need nothing from
 * MPI.  No MPI implementation is installed here, so this header lets those
 * files compile unmodified. */
#ifndef NBR_ORACLE_MPI_SHIM_H
#define NBR_ORACLE_MPI_SHIM_H
#endif
