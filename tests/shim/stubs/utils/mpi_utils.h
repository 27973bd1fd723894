// Stand-in for kiwi's utils/mpi_utils.h: the process record the reference's headers name.
#pragma once
namespace kiwi {
struct mpi_process {
  int own_rank = 0;
  int all_ranks = 1;
  int comm = 0;
};
}  // namespace kiwi
