// util.h -- error reporting shared by the host side of the library.
#pragma once
#include "ps_b200.h"

// Records msg as the thread's last error and returns code.
ps_status psb_fail(ps_status code, const char *msg);
// Records a CUDA error (with the failing call's name) and returns PS_ERR_CUDA.
ps_status psb_fail_cuda(int cuda_error, const char *what);
