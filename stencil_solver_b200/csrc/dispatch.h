// Internal step dispatch shared by the C ABI (capi.cu) and the run engine
// (run.cu): argument checks, kernel choice and tensor maps, with the full
// source descriptor (wavelet, device step counter, trace).
#pragma once

#include <string>

#include "kernels.h"
#include "stencil_b200.h"

namespace sb200 {

int dispatch_wave_f32(const float* p, const float* p_prev, const float* vel2, float* p_next,
                      const sb200_grid* grid, const SourceDesc& src, void* stream, bool exact);
// Two acoustic steps in one sweep (out1 = t+dt, out2 = t+2dt; w1 = the host
// sample of the second step).  outputs_may_alias: out1 == out2 is accepted
// (timing trials only: the values are then unusable).
int dispatch_wave2_f32(const float* p, const float* p_prev, const float* vel2, float* out1,
                       float* out2, const sb200_grid* grid, const SourceDesc& src, float w1,
                       void* stream, bool outputs_may_alias);
int dispatch_wave_f16(const uint16_t* p, uint16_t* p_prev_next, const uint16_t* k,
                      const sb200_grid* grid, const SourceDesc& src, const sb200_f16_scale* scale,
                      int phase, void* stream);
// Records msg as the calling thread's last error and returns code.
int set_error(int code, const std::string& msg);
// Address of the library's device error word on the current device (the word
// kernels record bounded-wait failures in), or nullptr if it cannot be looked up.
int* device_error_word();

}  // namespace sb200
