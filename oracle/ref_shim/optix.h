// Test infrastructure (oracle only): host stand-in for an OptiX header; see optixu/optixu_math_namespace.h.
#pragma once
#include <optixu/optixu_math_namespace.h>
