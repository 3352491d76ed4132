// Test-oracle shim (our code) standing in for the reference's Trilinos/Tpetra linear-system types
// in the golden-dump harness only (oracle/ref_harness.cpp, compiled with this directory first on
// its include path). The reference's Picard-Jacobian cell worker
// (solver/rdm/assembly/PGRDMPicardJacCellAssemblyWorker.hpp:444,454) hands its assembled entries
// to the system matrix and right-hand side through add_values(buffer); these classes record
// them, summed per (row, column) / row, instead of inserting them into a Tpetra matrix. No other
// part of the reference sees this header, and nothing here solves anything.
#ifndef PDEKIT_Linear_System_Tpetra_Fwd_hpp
#define PDEKIT_Linear_System_Tpetra_Fwd_hpp

#include <map>
#include <tuple>
#include <utility>
#include <vector>

#include "common/PDEKit.hpp"

namespace pdekit
{

namespace ls
{

template <typename Scalar, typename LocalOrdinal = int, typename GlobalOrdinal = long long,
          typename Node = void, const bool classic = false>
class TpetraCrsMatrix
{
  public:
  std::map<std::pair<Uint, Uint>, Scalar> entries;

  void add_values(const std::vector<std::tuple<Uint, Uint, Scalar>> &buffer)
  {
    for (const auto &t : buffer)
      entries[{std::get<0>(t), std::get<1>(t)}] += std::get<2>(t);
  }
};

template <typename Scalar, typename LocalOrdinal = int, typename GlobalOrdinal = long long,
          typename Node = void, const bool classic = false>
class TpetraMultiVector
{
  public:
  std::vector<Scalar> values;

  void add_values(const Uint column, const std::vector<std::tuple<Uint, Scalar>> &buffer)
  {
    (void)column;
    for (const auto &t : buffer)
    {
      if (std::get<0>(t) >= values.size())
        values.resize(std::get<0>(t) + 1, Scalar(0));
      values[std::get<0>(t)] += std::get<1>(t);
    }
  }
};

} // namespace ls

} // namespace pdekit

#endif
