/* MPI declarations for compiling the reference's gfind.c into the I/O
 * oracle (oracle/_ref/libgfref_io.so) without an MPI installation: types,
 * constants and unprototyped function declarations only.  Nothing in the
 * oracle calls gfind.c's main or any MPI function.  Test infrastructure
 * only. */
#ifndef GF_STUB_IO_MPI_H
#define GF_STUB_IO_MPI_H
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE; int MPI_TAG; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_LONG 2
#define MPI_LONG_LONG 3
#define MPI_FLOAT 4
#define MPI_BYTE 5
#define MPI_DOUBLE 6
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
int MPI_Init();
int MPI_Finalize();
int MPI_Comm_size();
int MPI_Comm_rank();
int MPI_Bcast();
int MPI_Send();
int MPI_Recv();
int MPI_Probe();
int MPI_Issend();
int MPI_Wait();
int MPI_Barrier();
#endif
