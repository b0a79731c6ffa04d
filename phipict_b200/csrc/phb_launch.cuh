// Host-side error reporting shared by the C ABI entry points: every entry point returns a
// phb_status code and leaves a message for phb_last_error(), instead of terminating the
// process as phiPICT's CUDA_CHECK_RETURN does (piso/device/launch.cuh:32-37).
#pragma once

#include <cuda_runtime.h>
#include <cstdio>
#include "../../include/phipict_b200.h"

namespace phb {

void setErrorText(const char *msg);

inline int setError(int code, const char *msg) {
	setErrorText(msg);
	return code;
}

inline int cudaStatus(cudaError_t e, const char *what) {
	if (e == cudaSuccess) return PHB_OK;
	char buf[512];
	snprintf(buf, sizeof(buf), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
	setErrorText(buf);
	return PHB_ERR_CUDA;
}

inline int checkLaunch(const char *what) { return cudaStatus(cudaGetLastError(), what); }

#define PHB_CUDA(call)                                               \
	do {                                                             \
		const int _st = ::phb::cudaStatus((call), #call);            \
		if (_st != PHB_OK) return _st;                               \
	} while (0)

} // namespace phb
