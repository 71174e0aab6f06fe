// Stand-in for deal.II/lac/trilinos_sparsity_pattern.h (declarations only).
#pragma once
namespace dealii::TrilinosWrappers
{
  class SparsityPattern
  {
  public:
    template <typename A, typename B, typename C, typename D>
    void
    reinit(const A &, const B &, const C &, const D &);
    void
    compress();
  };
} // namespace dealii::TrilinosWrappers
