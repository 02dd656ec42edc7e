// Test-infrastructure shim (oracle only). Stands in for the reference's
// NetCDF reader so that src/qes/Domain.cpp compiles without netCDF-C++.
// Only Domain's file constructor touches it, and the oracle never calls
// that constructor.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

struct NcVar {
  bool isNull() const { return true; }
};

class NetCDFInput {
public:
  explicit NetCDFInput(const std::string &) { throw std::runtime_error("NetCDF input is not available in the oracle build"); }
  void getDimensionSize(const std::string &, int &) {}
  template <typename T> void getVariableData(const std::string &, std::vector<T> &) {}
  void getVariable(const std::string &, NcVar &) {}
};
