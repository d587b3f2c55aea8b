// Stand-in for the cuda-api-wrappers constants header included by the reference's constants.hpp;
// the names it needs come from the api_wrappers.h stand-in beside it.
#pragma once
#include <cuda/api_wrappers.h>
