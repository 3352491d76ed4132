/* C++ host interface over the rds_b200 C ABI (rds_b200.h): RAII ownership of a context and
 * exceptions instead of status codes, for C++ hosts such as the pdekit drop-in solver
 * (pdekit_b200/GpuPGRDMethodExplicit.hpp). Header-only; C++14. */
#ifndef RDS_B200_HPP
#define RDS_B200_HPP

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "rds_b200.h"

namespace rds_b200
{

/* Raised for every status other than RDS_OK; status() is the C ABI code. */
class Error : public std::runtime_error
{
  public:
  Error(rds_status st, const std::string &msg) : std::runtime_error(msg), m_status(st)
  {
  }
  rds_status status() const
  {
    return m_status;
  }

  private:
  rds_status m_status;
};

inline const char *status_name(rds_status st)
{
  switch (st)
  {
  case RDS_OK:
    return "OK";
  case RDS_ERR_INVALID:
    return "INVALID";
  case RDS_ERR_CUDA:
    return "CUDA";
  case RDS_ERR_NONFINITE:
    return "NONFINITE";
  case RDS_ERR_NEG_PRESSURE:
    return "NEG_PRESSURE";
  case RDS_ERR_ITER_CAP:
    return "ITER_CAP";
  case RDS_ERR_UNSUPPORTED:
    return "UNSUPPORTED";
  case RDS_ERR_TOO_LARGE:
    return "TOO_LARGE";
  }
  return "?";
}

inline void check(rds_ctx *ctx, rds_status st, const char *what)
{
  if (st != RDS_OK)
    throw Error(st, std::string("rds_b200: ") + what + " failed (" + status_name(st) +
                        "): " + (ctx ? rds_last_error(ctx) : ""));
}

/* One solver context: the device copy of a mesh, its tables, weak conditions and fields. */
class Context
{
  public:
  explicit Context(const rds_desc &desc, void *stream = nullptr) : m_neq(desc.neq), m_nnodes(desc.nnodes)
  {
    rds_ctx *c = nullptr;
    const rds_status st = rds_create(&c, &desc, stream);
    m_ctx               = c;
    if (st != RDS_OK)
    {
      const std::string msg = c ? rds_last_error(c) : "";
      rds_destroy(c);
      m_ctx = nullptr;
      throw Error(st, std::string("rds_b200: rds_create failed (") + status_name(st) + "): " + msg);
    }
  }
  ~Context()
  {
    if (m_ctx)
      rds_destroy(m_ctx);
  }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;
  Context(Context &&o) noexcept : m_ctx(o.m_ctx), m_neq(o.m_neq), m_nnodes(o.m_nnodes)
  {
    o.m_ctx = nullptr;
  }
  Context &operator=(Context &&o) noexcept
  {
    std::swap(m_ctx, o.m_ctx);
    std::swap(m_neq, o.m_neq);
    std::swap(m_nnodes, o.m_nnodes);
    return *this;
  }

  rds_ctx *get() const
  {
    return m_ctx;
  }
  int neq() const
  {
    return m_neq;
  }
  int nnodes() const
  {
    return m_nnodes;
  }

  void add_cell_group(const rds_cell_group &g)
  {
    check(m_ctx, rds_add_cell_group(m_ctx, &g), "rds_add_cell_group");
  }
  void add_bc(const rds_bc_group &b)
  {
    check(m_ctx, rds_add_bc(m_ctx, &b), "rds_add_bc");
  }
  void finalize()
  {
    check(m_ctx, rds_finalize(m_ctx), "rds_finalize");
  }
  void set_option(const char *key, double value)
  {
    check(m_ctx, rds_set_option(m_ctx, key, value), "rds_set_option");
  }

  /* Nodal state, AoS [nnodes][neq]. */
  void set_state(const double *u_aos)
  {
    check(m_ctx, rds_set_state(m_ctx, u_aos), "rds_set_state");
  }

  /* Nodal stabilisation fields [nnodes] (nullptr removes one): the external blending
   * coefficient read by PGB cells, the artificial viscosity added by PGLDA cells. */
  void set_blending_coeff(const double *theta)
  {
    check(m_ctx, rds_set_blending_coeff(m_ctx, theta), "rds_set_blending_coeff");
  }
  void set_artificial_viscosity(const double *eps)
  {
    check(m_ctx, rds_set_artificial_viscosity(m_ctx, eps), "rds_set_artificial_viscosity");
  }
  void get_state(double *u_aos) const
  {
    check(m_ctx, rds_get_state(m_ctx, u_aos), "rds_get_state");
  }

  /* assemble_lhs_and_rhs(CFL) / assemble_rhs() / solve() of the explicit method. */
  void assemble(double cfl)
  {
    check(m_ctx, rds_assemble(m_ctx, cfl), "rds_assemble");
  }
  void assemble_rhs()
  {
    check(m_ctx, rds_assemble_rhs(m_ctx), "rds_assemble_rhs");
  }
  void update()
  {
    check(m_ctx, rds_update(m_ctx), "rds_update");
  }
  /* nsteps RK3TVD steps on the device (see rds_advance_rk3tvd). */
  void advance_rk3tvd(double cfl, int nsteps = 1)
  {
    check(m_ctx, rds_advance_rk3tvd(m_ctx, cfl, nsteps), "rds_advance_rk3tvd");
  }
  std::vector<double> residual_norm()
  {
    std::vector<double> n((size_t)m_neq);
    check(m_ctx, rds_residual_norm(m_ctx, n.data()), "rds_residual_norm");
    return n;
  }
  /* Any pointer may be null: residual AoS [nnodes][neq], dt, wave speed, dual volume [nnodes]. */
  void get_fields(double *res, double *dt, double *ws, double *vol) const
  {
    check(m_ctx, rds_get_fields(m_ctx, res, dt, ws, vol), "rds_get_fields");
  }

  struct IterateResult
  {
    int iterations = 0;
    bool reached   = false;
    std::vector<double> history; /* [iterations][neq] residual norms */
  };
  /* Device loop of assemble + solve to a residual drop (see rds_iterate). With
   * throw_on_cap = false an unreached drop is reported in `reached` instead of thrown. */
  IterateResult iterate(double cfl, int max_iter, double drop, bool throw_on_cap = true)
  {
    IterateResult r;
    r.history.resize((size_t)max_iter * (size_t)m_neq);
    const rds_status st = rds_iterate(m_ctx, cfl, max_iter, drop, &r.iterations, r.history.data());
    r.history.resize((size_t)r.iterations * (size_t)m_neq);
    r.reached = (st == RDS_OK);
    if (st != RDS_OK && !(st == RDS_ERR_ITER_CAP && !throw_on_cap))
      check(m_ctx, st, "rds_iterate");
    return r;
  }

  private:
  rds_ctx *m_ctx = nullptr;
  int m_neq      = 0;
  int m_nnodes   = 0;
};

} // namespace rds_b200

#endif
