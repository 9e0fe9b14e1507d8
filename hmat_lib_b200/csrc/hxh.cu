// HODLR x HODLR (placeholder until the device recompression lands).
#include "hxh.h"

namespace hb {

std::shared_ptr<DeviceTree> hxh_multiply(DeviceTree &, DeviceTree &, double, cudaStream_t,
                                         int *) {
  throw Error{INPUT_ERROR, "multiply_hodlr_hodlr: device path not built yet"};
}

}  // namespace hb
