// pf_api.h -- host-side helpers shared by the C-ABI entry points.
#pragma once
#include <cuda_runtime.h>

#include "../../include/pfoam.h"

// Records `msg` as this thread's last error and returns `code`.
int pf_fail(int code, const char* msg);
// Maps the last CUDA launch error (if any) to PF_ERR_CUDA.
int pf_check_launch(const char* where);
