// DeviceData.cuh -- the reference's sources include "DeviceData.cuh", which
// on its original (case-insensitive) file system is Core/include/devicedata.cuh.
// TEST INFRASTRUCTURE: this forwards to that header.
#pragma once
#include "devicedata.cuh"
