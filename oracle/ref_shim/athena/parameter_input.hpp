// Shim of Athena++ parameter_input.hpp: the two getters the EOS constructor
// uses, answering from a fixed table the harness fills.
#pragma once
#include <map>
#include <string>
#include "athena.hpp"

class ParameterInput {
 public:
  Real GetReal(const std::string &block, const std::string &name) {
    return vals.at(block + "/" + name);
  }
  Real GetOrAddReal(const std::string &block, const std::string &name, Real def) {
    auto it = vals.find(block + "/" + name);
    return it == vals.end() ? def : it->second;
  }
  std::map<std::string, Real> vals;
};
