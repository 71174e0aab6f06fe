// Stand-in for deal.II/lac/la_parallel_vector.h: a host vector whose local array holds every
// entry (one rank), with the members the adapter uses.
#pragma once
#include <cstddef>
#include <vector>

namespace dealii::LinearAlgebra::distributed
{
  template <typename Number>
  class Vector
  {
  public:
    using value_type     = Number;
    using iterator       = Number *;
    using const_iterator = const Number *;
    explicit Vector(const std::size_t n = 0)
      : values(n)
    {}
    iterator
    begin()
    {
      return values.data();
    }
    const_iterator
    begin() const
    {
      return values.data();
    }
    std::size_t
    locally_owned_size() const
    {
      return values.size();
    }
    void
    scale(const Vector &v)
    {
      for (std::size_t i = 0; i < values.size(); ++i)
        values[i] *= v.values[i];
    }

  private:
    std::vector<Number> values;
  };
} // namespace dealii::LinearAlgebra::distributed
