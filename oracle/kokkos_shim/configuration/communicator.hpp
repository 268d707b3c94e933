/*
 * configuration/communicator.hpp — single-process stand-in for CLEO's MPI/YAC communicator
 * (TEST INFRASTRUCTURE ONLY; replaces libs/configuration/communicator.hpp, which needs yaml-cpp,
 * MPI and YAC). Reports one process of rank 0.
 */
#pragma once
#include "mpi.h"
class init_communicator {
 public:
  static MPI_Comm get_communicator() { return MPI_COMM_WORLD; }
  static int get_yac_comp_id() { return -1; }
  static int get_comm_size() { return 1; }
  static int get_comm_rank() { return 0; }
};
