// Status strings and CUDA error bookkeeping of the C ABI.
#include "cp_common.h"

#include <cstdarg>
#include <cstdio>
#include <cstring>

namespace {
thread_local char t_last_error[256] = "";
}

cp_status cp_record_cuda_error(cudaError_t e, cp_status status) {
    std::snprintf(t_last_error, sizeof(t_last_error), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
    return status;
}

cp_status cp_fail(cp_status status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(t_last_error, sizeof(t_last_error), fmt, ap);
    va_end(ap);
    return status;
}

cp_status cp_check_launch() {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return CP_OK;
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return cp_record_cuda_error(e, CP_ERR_NO_DEVICE);
    if (e == cudaErrorMemoryAllocation) return cp_record_cuda_error(e, CP_ERR_NOMEM);
    return cp_record_cuda_error(e, CP_ERR_CUDA);
}

extern "C" {

const char* cp_status_string(int status) {
    switch (status) {
    case CP_OK: return "ok";
    case CP_ERR_INVALID: return "invalid argument";
    case CP_ERR_CUDA: return "CUDA runtime error";
    case CP_ERR_NOMEM: return "device allocation failed";
    case CP_ERR_CAPACITY: return "worklist capacity exceeded";
    case CP_ERR_DEVICE: return "device-side error flag raised";
    case CP_ERR_TRAP_SITE: return "a box reached a reference trap site";
    case CP_ERR_NOFIT: return "fit check fired where the reference traps";
    case CP_ERR_INTERRUPTED: return "interrupted";
    case CP_ERR_NOT_PROVED: return "not proved within the limits";
    case CP_ERR_NO_DEVICE: return "no usable CUDA device";
    }
    return "unknown status";
}

const char* cp_last_error_string(void) { return t_last_error; }

const char* cp_version(void) { return "circlepacking_b200 0.1 (sm_100a)"; }
}
