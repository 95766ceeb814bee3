// Factorised sparse approximate inverse on the IC(0) block pattern (fsai.cu).
#pragma once

#include "cipc_internal.h"

namespace cipc {

// Builds G into c.mpGS / c.mpGD for the current system; needs the scaling
// and mirror slots of mpnnPrepare(c, false).
void fsaiBuild(Ctx& c);

}  // namespace cipc
