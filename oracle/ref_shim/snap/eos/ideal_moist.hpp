// Shim of snapy's IdealMoist equation of state and of the kintera tables
// that canoe src/interface/eos.hpp reads.  get_gamma (eos.hpp:48-67) needs
// the cv and inverse molecular-weight ratio tables and the vapour / cloud
// counts; get_rd / get_gammad (eos.hpp:14-21) need the gas constant, the
// dry molecular weight and the dry cv / R.  The harness fills them from the
// same parameters the oracle and the kernels take.
#pragma once
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <torch/torch.h>
#include <snap/snap.h>

namespace kintera {
namespace constants {
inline double Rgas = 8.314462618;
}
inline std::vector<double> species_weights;  // [0] = dry molecular weight
inline std::vector<double> species_cref_R;   // [0] = dry cv / R

struct ThermoOptions {
  std::vector<int> vapor_ids_, cloud_ids_;
  const std::vector<int> &vapor_ids() const { return vapor_ids_; }
  const std::vector<int> &cloud_ids() const { return cloud_ids_; }
};
struct ThermoYImpl {
  ThermoOptions options;
};
}  // namespace kintera

namespace snap {
class IdealMoistImpl {
 public:
  std::shared_ptr<kintera::ThermoYImpl> pthermo;
  torch::Tensor cv_ratio_m1, inv_mu_ratio_m1;
  torch::Tensor compute(const std::string &, const std::vector<torch::Tensor> &) {
    throw std::runtime_error("snapy conversions are not part of the pin");
  }
  torch::Tensor f_sig(const torch::Tensor &) {
    throw std::runtime_error("snapy conversions are not part of the pin");
  }
};

// torch::nn::ModuleHolder-like handle
class IdealMoist {
 public:
  IdealMoist(std::shared_ptr<IdealMoistImpl> p) : p_(std::move(p)) {}
  IdealMoistImpl *operator->() const { return p_.get(); }

 private:
  std::shared_ptr<IdealMoistImpl> p_;
};
}  // namespace snap
