/*
 * mpi.h — declarations-only stand-in for the MPI calls that CLEO's hot-path sources name
 * (TEST INFRASTRUCTURE ONLY). The oracle's reference build runs one process, where the reference
 * never reaches these calls (cartesian_transport_across_domain.cpp:32-39); each one throws if it
 * is reached.
 */
#pragma once
#include <stdexcept>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_UNSIGNED 3
#define MPI_UNSIGNED_LONG 4
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
[[noreturn]] inline int cleo_shim_mpi_unreachable() { throw std::runtime_error("MPI call reached in single-process oracle build"); }
inline int MPI_Alltoall(const void*, int, MPI_Datatype, void*, int, MPI_Datatype, MPI_Comm) { cleo_shim_mpi_unreachable(); }
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { cleo_shim_mpi_unreachable(); }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { cleo_shim_mpi_unreachable(); }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { cleo_shim_mpi_unreachable(); }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
