// Stand-in for DP3's base/DPBuffer.h (which needs casacore) with the part the
// regular SolveData constructor reads (ddecal/gain_solvers/SolveData.cc:
// 77-188): named visibility cubes [baseline][channel][correlation] of
// complex<float> ("" is the data, other names are model directions) and an
// optional weight cube of the same shape. Only for building DP3's sources
// outside a DP3 tree; a DP3 build uses the real DPBuffer.
#ifndef DP3B200_STANDIN_BASE_DPBUFFER_H
#define DP3B200_STANDIN_BASE_DPBUFFER_H

#include <complex>
#include <map>
#include <stdexcept>
#include <string>

#include <xtensor/containers/xtensor.hpp>

namespace dp3::base {

class DPBuffer {
 public:
  using DataType = xt::xtensor<std::complex<float>, 3>;
  using WeightsType = xt::xtensor<float, 3>;

  DPBuffer() = default;
  DPBuffer(DPBuffer&&) noexcept = default;
  DPBuffer& operator=(DPBuffer&&) noexcept = default;

  // Adds (or resizes) the cube `name`: [n_baselines][n_channels][n_corr].
  DataType& AddData(const std::string& name, size_t n_baselines, size_t n_channels,
                    size_t n_corr) {
    DataType& d = data_[name];
    d.resize({n_baselines, n_channels, n_corr});
    return d;
  }
  bool HasData(const std::string& name = "") const { return data_.count(name) != 0; }
  DataType& GetData(const std::string& name = "") { return Find(name); }
  const DataType& GetData(const std::string& name = "") const {
    return const_cast<DPBuffer*>(this)->Find(name);
  }
  WeightsType& GetWeights() { return weights_; }
  const WeightsType& GetWeights() const { return weights_; }

 private:
  DataType& Find(const std::string& name) {
    auto it = data_.find(name);
    if (it == data_.end()) throw std::runtime_error("DPBuffer has no data named '" + name + "'");
    return it->second;
  }

  std::map<std::string, DataType> data_;
  WeightsType weights_;
};

}  // namespace dp3::base

#endif
