// Stand-in for deal.II/lac/la_parallel_block_vector.h.
#pragma once
#include <deal.II/lac/la_parallel_vector.h>
namespace dealii::LinearAlgebra::distributed
{
  template <typename Number>
  class BlockVector
  {};
} // namespace dealii::LinearAlgebra::distributed
