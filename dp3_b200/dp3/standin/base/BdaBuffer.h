// Stand-in for DP3's base/BdaBuffer.h (which needs casacore): DP3's
// BdaSolverBuffer.h only holds BdaBuffer objects by std::unique_ptr in the
// declarations that SolveData.cc reads, so an empty class suffices to compile
// SolveData.cc. Only for building DP3's sources outside a DP3 tree.
#ifndef DP3B200_STANDIN_BASE_BDABUFFER_H
#define DP3B200_STANDIN_BASE_BDABUFFER_H

namespace dp3::base {
class BdaBuffer {};
}  // namespace dp3::base

#endif
