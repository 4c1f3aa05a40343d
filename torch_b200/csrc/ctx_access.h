// Read access to a context's parameters and device pointers for entry points
// that live outside capi.cu.
#pragma once
#include <string>

#include "../../include/torch_b200.h"
#include "trg_types.h"

namespace trg {
const Params& ctx_params(const trg_ctx* c);
State ctx_state(const trg_ctx* c);
int ctx_device(const trg_ctx* c);
int ctx_fp32_zchunk(const trg_ctx* c);
int ctx_fail(trg_ctx* c, int code, const std::string& msg);
}  // namespace trg
