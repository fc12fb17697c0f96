// See cuda_libs_stub.h: test-infrastructure stand-in, CPU build of the reference only.
#pragma once
#include "cuda_libs_stub.h"
