// Test harness: the device float math restatements (psy_libm.cuh) compiled
// for the host, so a CPU test can hold them against the host C library.
#include "psy_libm.cuh"

extern "C" int libm_restated(int fn, unsigned n, const float* x, float* out) {
	for (unsigned i = 0; i < n; ++i) {
		switch (fn) {
			case 0: out[i] = lm_sinf(x[i]); break;
			case 1: out[i] = lm_cosf(x[i]); break;
			case 2: out[i] = lm_acosf(x[i]); break;
			case 3: out[i] = lm_asinf(x[i]); break;
			case 4: out[i] = lm_expf(x[i]); break;
			default: return -1;
		}
	}
	return 0;
}
