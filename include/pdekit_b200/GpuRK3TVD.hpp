#ifndef PDEKIT_B200_GPU_RK3TVD_HPP
#define PDEKIT_B200_GPU_RK3TVD_HPP

/* Drop-in for pdekit's time::RK3TVD (src/solver/time/ExplicitTimeStepper.hpp, .cpp:46-100).
 *
 * A program that advances its solver through an ExplicitTimeStepperBase constructs GpuRK3TVD
 * instead of RK3TVD. Given a GpuPGRDMethodExplicit, advance_in_time runs the three stages on
 * the device in one graph launch (rds_advance_rk3tvd) and refreshes the solver's solution,
 * residual and time-step functions once; given any other solver it runs the reference's own
 * RK3TVD, so the same program works with either solver. */

#include "GpuPGRDMethodExplicit.hpp"
#include "solver/time/ExplicitTimeStepper.hpp"

namespace pdekit
{

namespace solver
{

namespace time
{

class GpuRK3TVD : public ExplicitTimeStepperBase
{
  public:
  void setup(const Uint nb_fields, const Uint nb_entries) override
  {
    m_host.setup(nb_fields, nb_entries);
  }

  void advance_in_time(SolverBase &solver, const Real CFL) override
  {
    if (auto *dev = dynamic_cast<rdm::DeviceRK3TVDSolver *>(&solver))
      dev->advance_rk3tvd(CFL, 1);
    else
      m_host.advance_in_time(solver, CFL);
  }

  private:
  RK3TVD m_host;
};

} // namespace time

} // namespace solver

} // namespace pdekit

#endif
