// Stand-in for schaapcommon's RecursiveFor: in DP3 its existence lets a
// StaticFor run inside another; the stand-in pool always allows that (nested
// parallel loops get their own threads), so this object carries no state.
// Only for building DP3's sources outside a DP3 tree.
#ifndef DP3B200_STANDIN_SCHAAPCOMMON_THREADING_RECURSIVEFOR_H
#define DP3B200_STANDIN_SCHAAPCOMMON_THREADING_RECURSIVEFOR_H

#include "staticfor.h"
#include "threadpool.h"

namespace schaapcommon {

class RecursiveFor {
 public:
  RecursiveFor() = default;
  RecursiveFor(const RecursiveFor&) = delete;
  RecursiveFor& operator=(const RecursiveFor&) = delete;
};

}  // namespace schaapcommon

#endif
