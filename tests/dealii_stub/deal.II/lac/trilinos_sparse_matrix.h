// Stand-in for deal.II/lac/trilinos_sparse_matrix.h (declarations only).
#pragma once
#include <deal.II/lac/trilinos_sparsity_pattern.h>
namespace dealii::TrilinosWrappers
{
  class SparseMatrix
  {
  public:
    void
    reinit(const SparsityPattern &);
  };
} // namespace dealii::TrilinosWrappers
