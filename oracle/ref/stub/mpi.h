/* Minimal MPI declarations so the reference's hot-path translation units
 * compile without an MPI installation.  None of the compiled functions calls
 * MPI; subhaloden.mod6.c and tsc_omp2.c only include the header.
 * Test infrastructure only: used by the oracle/_ref build recipe. */
#ifndef GF_STUB_MPI_H
#define GF_STUB_MPI_H
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef struct { int MPI_SOURCE; int MPI_TAG; } MPI_Status;
#define MPI_LONG_LONG 0
#define MPI_LONG 0
#endif
