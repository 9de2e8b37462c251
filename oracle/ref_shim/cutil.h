// cutil.h -- host stand-in for the CUDA SDK utility header the reference's
// kernel files include (TEST INFRASTRUCTURE): the error-check macros pass
// the call through.
#pragma once
#define CUDA_SAFE_CALL(call) (call)
#define CUT_SAFE_CALL(call) (call)
#define CUT_CHECK_ERROR(msg)
