/*
 * mpdg_heat_dealii.hpp - MeltPoolDG-side binding of the B200 heat operator (header only,
 * C++20, compiled inside MeltPoolDG next to source/heat/heat_diffuse_operator.cpp).
 *
 * HeatDiffuseOperatorB200<3> derives from MeltPoolDG::OperatorMatrixFree<3, double>
 * (include/meltpooldg/core/operator_base.hpp:188-282) and forwards its verbs to the C ABI of
 * mpdg_heat.h. Its VectorType is the base's, the host vector
 * dealii::LinearAlgebra::distributed::Vector<double> (operator_base.hpp:192): on one MPI rank
 * the local array holds every DoF, in deal.II's numbering, so the verbs are the *_host entry
 * points and the constructor passes the map from deal.II's DoF numbering to the library's
 * lexicographic one (mpdg_heat_set_dof_permutation).
 *
 * What the base does not make virtual:
 *  - OperatorBase::reset_time_increment (operator_base.hpp:41-46) stores dt and 1/dt in the
 *    base; the adapter forwards the stored value to the library before each verb.
 *  - HeatDiffuseOperation holds a std::unique_ptr<HeatDiffuseMultiPhaseOperator<dim, number>>
 *    (heat_diffuse_operation.hpp:84), whose vmult/pre/post are final; the operation's member
 *    type has to become OperatorMatrixFree<dim, number> to hold this adapter (the patch is
 *    written out beside this header's documentation).
 *
 * Like HeatDiffuseMultiPhaseOperator, the operator keeps references to the operation's
 * temperature, temperature_old and heat_source vectors (heat_diffuse_operator.hpp:128-135);
 * pre() uploads the linearisation point (pre() is called before create_rhs and before each
 * linear solve, heat_diffuse_operation.cpp:89, :237, :275).
 * Errors: a non-zero status becomes the deal.II exception MeltPoolDG throws at that point
 * (ExcZeroTimeIncrement for a zero time increment, ExcMessage with the library's message
 * otherwise).
 */
#pragma once

#include <meltpooldg/core/exceptions.hpp>
#include <meltpooldg/core/operator_base.hpp>

#include <cstdint>
#include <string>
#include <vector>

#include "mpdg_heat.h"

namespace MeltPoolDG::Heat
{
  template <int dim>
  class HeatDiffuseOperatorB200 : public OperatorMatrixFree<dim, double>
  {
    static_assert(dim == 3, "the B200 heat operator runs on 3D hexahedral box meshes");

  public:
    using VectorType = typename OperatorMatrixFree<dim, double>::VectorType;

    /**
     * mesh, material: the structured box and the law (mpdg_heat.h); lex_of_dof[i]: the
     * lexicographic index of deal.II DoF i (empty: the numbers already agree).
     */
    HeatDiffuseOperatorB200(const mpdg_mesh_desc            &mesh,
                            const mpdg_material             &material,
                            const std::vector<std::int64_t> &lex_of_dof,
                            const VectorType                &temperature_in,
                            const VectorType                &temperature_old_in,
                            const VectorType                &heat_source_in,
                            const int                        device = 0)
      : temperature(temperature_in)
      , temperature_old(temperature_old_in)
      , heat_source(heat_source_in)
    {
      check(mpdg_heat_create(&mesh, device, &handle));
      check(mpdg_heat_set_material(handle, &material));
      std::int64_t n = 0;
      check(mpdg_heat_n_dofs(handle, &n));
      n_dofs = n;
      if (!lex_of_dof.empty())
        {
          AssertThrow(static_cast<std::int64_t>(lex_of_dof.size()) == n_dofs,
                      dealii::ExcMessage("the DoF map must have one entry per DoF"));
          check(mpdg_heat_set_dof_permutation(handle, lex_of_dof.data()));
        }
    }

    ~HeatDiffuseOperatorB200() override
    {
      mpdg_heat_destroy(handle);
    }

    HeatDiffuseOperatorB200(const HeatDiffuseOperatorB200 &) = delete;
    HeatDiffuseOperatorB200 &
    operator=(const HeatDiffuseOperatorB200 &) = delete;

    void
    pre() override
    {
      sync_time_increment();
      check_size(temperature);
      check_size(temperature_old);
      check(mpdg_heat_set_linearization_host(handle, temperature.begin(), temperature_old.begin()));
    }

    void
    post() override
    {}

    void
    reinit() override
    {}

    void
    vmult(VectorType &dst, const VectorType &src) const override
    {
      sync_time_increment();
      check_size(dst);
      check_size(src);
      check(mpdg_heat_vmult_host(handle, dst.begin(), src.begin()));
    }

    void
    create_rhs(VectorType &dst, const VectorType &src) const override
    {
      sync_time_increment();
      check_size(dst);
      check_size(src);
      check_size(heat_source);
      check(mpdg_heat_create_rhs_host(handle, dst.begin(), src.begin(), heat_source.begin()));
    }

    void
    compute_inverse_diagonal_from_matrixfree(VectorType &diag) const override
    {
      sync_time_increment();
      check_size(diag);
      check(mpdg_heat_compute_inverse_diagonal_host(handle, diag.begin()));
    }

    /** The library handle, for the device-side solvers (mpdg_heat_linear_solve, time step). */
    mpdg_heat *
    native_handle() const
    {
      return handle;
    }

  private:
    void
    sync_time_increment() const
    {
      // an increment never set (numbers::invalid_double) reaches the library as zero, which
      // it reports as MPDG_ERR_ZERO_TIME_INCREMENT at the next verb that needs it
      const double dt = numbers::is_invalid(this->time_increment) ? 0.0 : this->time_increment;
      if (dt != applied_time_increment)
        {
          check(mpdg_heat_reset_time_increment(handle, dt));
          applied_time_increment = dt;
        }
    }

    void
    check_size(const VectorType &v) const
    {
      AssertThrow(static_cast<std::int64_t>(v.locally_owned_size()) == n_dofs,
                  dealii::ExcMessage("the B200 operator owns every DoF on one rank"));
    }

    static void
    check(const int status)
    {
      if (status == MPDG_ERR_ZERO_TIME_INCREMENT)
        AssertThrowZeroTimeIncrement(0.0);
      AssertThrow(status == MPDG_OK,
                  dealii::ExcMessage("mpdg_heat status " + std::to_string(status) + ": " +
                                     mpdg_last_error()));
    }

    mpdg_heat                   *handle = nullptr;
    std::int64_t                 n_dofs = 0;
    mutable double               applied_time_increment = 0.0;
    const VectorType            &temperature;
    const VectorType            &temperature_old;
    const VectorType            &heat_source;
  };
} // namespace MeltPoolDG::Heat
