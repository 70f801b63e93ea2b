// Status codes shared by host and device code (the C ABI mirrors them as
// IGR_ERR_* in include/instantgr_b200.h).
#pragma once

namespace igr {

enum : int {
    OK = 0,
    ERR_INVALID = -1,
    ERR_IO = -2,
    ERR_FORMAT = -3,
    ERR_CUDA = -4,
    ERR_CAPACITY = -5,
    ERR_TIMEOUT = -6,
    ERR_STATE = -7,
};

}  // namespace igr
