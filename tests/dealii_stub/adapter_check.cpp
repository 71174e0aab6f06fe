// Compiles the reference-side adapter (include/mpdg_heat_dealii.hpp) against MeltPoolDG's own
// operator_base.hpp and preconditioner_jacobi.hpp, with deal.II replaced by the stand-ins of
// this directory, and checks that it is a complete OperatorMatrixFree<3, double> that the
// reference's Jacobi preconditioner accepts.
#include <meltpooldg/core/operator_base.hpp>
#include <meltpooldg/linear_algebra/preconditioner_jacobi.hpp>

#include <mpdg_heat_dealii.hpp>

#include <memory>
#include <type_traits>

using Adapter    = MeltPoolDG::Heat::HeatDiffuseOperatorB200<3>;
using Base       = MeltPoolDG::OperatorMatrixFree<3, double>;
using VectorType = Base::VectorType;

static_assert(std::is_base_of_v<Base, Adapter>);
static_assert(std::is_same_v<Adapter::VectorType, dealii::LinearAlgebra::distributed::Vector<double>>);
static_assert(!std::is_abstract_v<Adapter>);
static_assert(MeltPoolDG::JacobiPreconditionerOperatorType<Adapter, VectorType>);
static_assert(MeltPoolDG::JacobiPreconditionerOperatorType<Base, VectorType>);

// the calls HeatDiffuseOperation makes through its operator member once that member is an
// OperatorMatrixFree<dim, number> (heat_diffuse_operation.cpp:89-96, :217, :237-246, :275-295)
void
drive(std::unique_ptr<Base> &op, VectorType &rhs, VectorType &x, const VectorType &old)
{
  op->reset_time_increment(1e-3);
  op->pre();
  op->create_rhs(rhs, old);
  op->vmult(x, rhs);
  op->compute_inverse_diagonal_from_matrixfree(x);
  op->post();
}

std::unique_ptr<Base>
make(const mpdg_mesh_desc &mesh, const mpdg_material &mat, const VectorType &T,
     const VectorType &T_old, const VectorType &q)
{
  return std::make_unique<Adapter>(mesh, mat, std::vector<std::int64_t>{}, T, T_old, q);
}
