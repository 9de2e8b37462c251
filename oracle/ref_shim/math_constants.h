// math_constants.h -- host stand-in (TEST INFRASTRUCTURE).
#pragma once
#define CUDART_PI_F 3.141592654f
#define CUDART_INF_F __builtin_inff()
