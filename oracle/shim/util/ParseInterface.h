// Test-infrastructure shim (oracle only). The reference's ParseInterface
// reads XML through Boost.PropertyTree, which this image does not have.
// The building classes only call parsePrimitive from parseValues(); here it
// reads the named value from a table the oracle driver fills before it calls
// parseValues(), so that the reference's own parseValues() and everything
// after it run unchanged.
#pragma once
// the standard headers the reference's ParseInterface.h brings in, which the
// building headers rely on
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

class ParseInterface {
public:
  virtual ~ParseInterface() = default;

  // name -> value for the next parseValues() call
  static std::map<std::string, double> &shimValues()
  {
    static std::map<std::string, double> v;
    return v;
  }

  template <typename T>
  void parsePrimitive(bool required, T &out, const std::string &name)
  {
    auto it = shimValues().find(name);
    if (it != shimValues().end()) out = static_cast<T>(it->second);
    else if (required) throw std::runtime_error("oracle shim: no value for " + name);
  }
};
