/* Stand-in for <mpi.h> where the compatibility layer is built without an MPI
 * installation: the communicator type that src/fluforces/imp.h names and
 * the two cartesian-topology queries fluforces_halo_ini makes (standard MPI
 * signatures).  A real uDeviceX build uses its MPI; the driver
 * ctc_b200/compat/udx_drive.cpp defines them for one periodic rank. */
#pragma once
typedef struct ctc_compat_check_comm *MPI_Comm;
int MPI_Cart_get(MPI_Comm comm, int maxdims, int dims[], int periods[], int coords[]);
int MPI_Cart_rank(MPI_Comm comm, const int coords[], int *rank);
