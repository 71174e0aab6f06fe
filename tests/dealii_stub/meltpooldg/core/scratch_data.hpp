// Stand-in for MeltPoolDG's core/scratch_data.hpp (whose real version includes deal.II's
// MatrixFree): the ScratchData members operator_base.hpp and preconditioner_jacobi.hpp name.
#pragma once
#include <deal.II/base/mpi.h>

namespace MeltPoolDG
{
  template <int dim, int spacedim = dim, typename number = double>
  class ScratchData
  {
  public:
    MPI_Comm
    get_mpi_comm(const unsigned int = 0) const;
    const int &
    get_locally_owned_dofs(const unsigned int) const;
    const int &
    get_locally_relevant_dofs(const unsigned int) const;
    const int &
    get_dof_handler(const unsigned int) const;
    const int &
    get_constraint(const unsigned int) const;
    template <typename VectorType>
    void
    initialize_dof_vector(VectorType &, const unsigned int) const;
  };
} // namespace MeltPoolDG
