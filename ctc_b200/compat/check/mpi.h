/* Stand-in for <mpi.h> where the compatibility layer is only compile-checked
 * against the reference's headers (no MPI installation): the communicator
 * type that src/fluforces/imp.h names.  A real uDeviceX build uses its MPI. */
#pragma once
typedef struct ctc_compat_check_comm *MPI_Comm;
