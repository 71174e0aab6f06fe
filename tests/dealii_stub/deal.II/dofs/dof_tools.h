// Stand-in for deal.II/dofs/dof_tools.h (declaration only).
#pragma once
namespace dealii::DoFTools
{
  template <typename DoFHandlerType, typename SparsityType, typename ConstraintsType>
  void
  make_sparsity_pattern(const DoFHandlerType &,
                        SparsityType &,
                        const ConstraintsType &,
                        bool,
                        unsigned int);
} // namespace dealii::DoFTools
