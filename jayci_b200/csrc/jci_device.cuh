// jci_device.cuh -- device-side state and helpers shared by the CUDA units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "jci_internal.h"

namespace jci {

#define JCI_CUDA(call)                                            \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

jci_status cuda_fail(cudaError_t e, const char *what, const char *file, int line);

// Raise a kernel's dynamic shared-memory cap to the device's opt-in maximum.
// The cap is an attribute of the function in the context, shared by every
// host thread: setting it to one launch's own size would shrink it under a
// concurrent launch of the same kernel for a larger space (solve server).
template <typename K>
inline cudaError_t smem_optin(K kern) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // the opt-in limit covers the kernel's static shared memory too
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - (int)fa.sharedSizeBytes);
    return e;
}

// Packed excitation entry.
//   x: bits 0..29 target string, bit 31 set for a negative phase
//   y (single): io | fo << 8 | pair << 16   (pair = packed index of (io,fo))
//   y (double): io0 | fo0 << 8 | io1 << 16 | fo1 << 24
// Orbitals are 1-based CI orbital numbers (< 256).
struct SpinTables {
    int nstr = 0, nelec = 0, ngrp = 0;
    int *istr = nullptr;           // nstr x nelec
    int *grp = nullptr;            // group of each string
    int *gstart = nullptr;         // per group
    int *gnstr = nullptr;
    long long *soff = nullptr, *doff = nullptr;  // nstr + 1
    uint2 *sing = nullptr, *doub = nullptr;
    double *a1 = nullptr;          // one-body part of each single (no phase)
    float *a1f = nullptr;
    double *eself = nullptr;       // same-spin diagonal energy of each string
    int max_sing = 0, max_doub = 0;
    long long nsing = 0, ndoub = 0;
    // dense tables for single-group (FCI/CAS) spaces
    uint32_t *fsing = nullptr;     // [e][nstr] target | sign << 31
    uint16_t *fspair = nullptr;    // [e][nstr] pair index
    uint64_t *occ = nullptr;       // occupation bit mask of internal orbitals
};

struct DeviceState {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evin = nullptr, evout = nullptr;  // ordering with the legacy default stream
    float last_sigma_ms = 0.f;
    SpinTables t[2];
    int npq = 0;
    int *pairidx = nullptr;        // pegrps x qegrps
    long long *pqoff = nullptr;    // npq + 1
    int norb = 0, npair = 0;
    long long m2len = 0;
    double *m1 = nullptr, *m2 = nullptr;
    float *m1f = nullptr, *m2f = nullptr;
    double *hd = nullptr;          // <i|H|i>
    float *hdf = nullptr;
    bool single_group = false;
    int *pqg = nullptr;            // npq x 2 group pair of each block
    void *io_v = nullptr, *io_s = nullptr;  // host-API staging buffers
    size_t io_bytes = 0;
    struct FciTables *fci = nullptr;   // single-group fast path (jci_fci.cu)
    struct DavidsonBuffers *dav = nullptr;  // jci_davidson.cu
    // Device flag read by every sigma kernel at entry: when nonzero the
    // kernel returns at once.  Set while a Davidson iteration is captured
    // into a CUDA graph, so that iterations launched after the solve has
    // stopped cost no sigma work; null otherwise.
    const int *sigma_skip = nullptr;
};

// Kernel-facing view of a space (POD, passed by value).
struct SpaceView {
    long long ndets;
    const int *skip;  // DeviceState::sigma_skip
    int npq, qegrps, norb, npair;
    const long long *pqoff;
    const int *pairidx;
    const int *pqg;
    struct Spin {
        int nstr, nelec;
        const int *istr, *grp, *gstart, *gnstr;
        const long long *soff, *doff;
        const uint2 *sing, *doub;
    } a, b;
};

SpaceView make_view(const DeviceState *d);

__host__ __device__ inline int pair_index(int p, int q) {  // 1-based orbitals
    int hi = p > q ? p : q, lo = p > q ? q : p;
    return hi * (hi - 1) / 2 + lo - 1;
}

__host__ __device__ inline long long eri_index(int pa, int pb) {  // 0-based pairs
    long long hi = pa > pb ? pa : pb, lo = pa > pb ? pb : pa;
    return hi * (hi + 1) / 2 + lo;
}

}  // namespace jci
