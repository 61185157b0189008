// jci_kernels.cuh -- entry points between the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include "jci_device.cuh"

namespace jci {

// FCI / CAS fast path (single electron-occupation group per spin), jci_fci.cu.
bool fci_supported(const jci_space *s);
jci_status fci_prepare(jci_space *s);
jci_status fci_sigma(jci_space *s, int nvec, const void *v, void *sig, long long ld,
                     int precision, cudaStream_t st);
void fci_free(DeviceState *d);
void fci_tuning(const jci_space *s, int precision, int *mode, int *nt, int *R, int *B,
                float *ms);
jci_status fci_force_plan(jci_space *s, int precision, int mode, int nt, int R, int B);
jci_status fci_sigma_noalloc(jci_space *s, const void *v, void *o, int precision,
                             cudaStream_t st);
size_t fci_noalloc_scratch_bytes();

// Generic path (any truncated space), jci_device.cu.
jci_status device_sigma_generic(jci_space *s, int nvec, const void *vin, void *sout,
                                long long ld, int precision, cudaStream_t st);

// Davidson buffers (jci_davidson.cu).
void davidson_free(DeviceState *d);

}  // namespace jci
