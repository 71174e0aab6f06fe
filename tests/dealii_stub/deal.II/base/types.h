// Stand-in for deal.II/base/types.h.
#pragma once
namespace dealii
{
  namespace types
  {
    using boundary_id          = unsigned int;
    using global_dof_index     = unsigned long long;
  } // namespace types
  namespace numbers
  {
    constexpr unsigned int invalid_unsigned_int = static_cast<unsigned int>(-1);
  } // namespace numbers
} // namespace dealii
