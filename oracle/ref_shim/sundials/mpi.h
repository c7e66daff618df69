/* TEST INFRASTRUCTURE ONLY: the MPI names the reference's CiPA bench uses,
 * for one process (rank 0 of 1). */
#ifndef CEP_STUB_MPI_H
#define CEP_STUB_MPI_H
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);
#endif
