// jci_kernels.cuh -- entry points between the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "jci_device.cuh"

namespace jci {

// FCI / CAS fast path (single electron-occupation group per spin), jci_fci.cu.
bool fci_supported(const jci_space *s);
// JCI_ERR_TIMEOUT (and the flag cleared) if a product kernel's bounded
// device wait expired since the last call; synchronises with the device.
jci_status fci_wait_status(jci_space *s);
// Test hook: the next launch of the shared-panel product leaves the GEMM
// items of its first rows undone, so that its gathers' waits expire.
jci_status fci_arm_wait_expiry(jci_space *s);
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

// Alpha-single x beta-single part of the one-group sigma as one fused
// kernel (product chunks in shared memory), jci_fci_ab.cu.
template <typename T>
struct AbArgs {
    int na, nb, sa, npair, mrows, nchunk;
    int offs, maxent;       // row stride of off; longest (padded) chunk list
    int vec;                // 16-byte copies of C rows (nb even, C 16-byte aligned)
    const uint32_t *fsA;    // [single][Ia] target | phase << 31
    const uint16_t *fpA;    // [single][Ia] pair index
    const T *a1A;           // [single][Ia] one-body part
    const T *m2;            // packed (pq|rs)
    const uint16_t *off;    // [chunk][offs] entry offsets within the chunk
    const uint32_t *base;   // [chunk + 1] first entry of each chunk (multiples of 4)
    const uint32_t *ent;    // col | row << 8 | phase << 31
    const int *skip;        // nonzero: return at once
};
struct AbTables {
    int tx = 0, nchunk = 0, offs = 0, maxent = 0;
    uint16_t *off = nullptr;
    uint32_t *base = nullptr, *ent = nullptr;
};
struct AbShape {
    int nb, sa, sb, nelb, npair;   // beta strings, singles per string, beta electrons
};
size_t ab_smem(const AbShape &sh, int tx, size_t w);
bool ab_possible(const AbShape &sh, int tx, size_t w, size_t smem_max);
jci_status ab_tables_build(const jci_space *s, int npair, int tx, AbTables *t);
void ab_tables_free(AbTables *t);
template <typename T>
jci_status ab_launch(const AbArgs<T> &a, int tx, int device, const T *v, T *o,
                     cudaStream_t st);
// The FP32 fused product on tcgen05 tensor cores (jci_fci_tc.cu), chunk width
// cw = 32 or 64 (the entry lists of tx = cw / 4).  status (device int,
// nullable) is set to 1 if a bounded wait of the kernel expired.
size_t tc_smem(const AbShape &sh, int cw);
bool tc_possible(const AbShape &sh, int cw, size_t smem_max);
jci_status tc_launch(const AbArgs<float> &a, int cw, int device, const float *v, float *o,
                     int *status, cudaStream_t st);

// Same-spin doubles over groups of consecutive strings, jci_fci_group.cu.
constexpr int kGroupRows = 16;
template <typename T>
struct GroupArgs {
    int rows, len;          // output rows (strings of the spin) x row length
    const int *uoff;        // [group + 1] first union entry of each group
    const int *uidx;        // union entries: source rows
    const int *useg;        // [group][17] class boundaries (class q: row quads q)
    const T *coef;          // [entry][kGroupRows] double values (0: not reached)
    const T *hd;            // [row][column] diagonal, or null
    int add;                // 1: Y += result, 0: Y = result
    const int *skip;        // nonzero: return at once
};
struct GroupTables {
    int ng = 0, rows = 0, nd = 0;
    size_t nu = 0;          // union entries over all groups
    int *uoff = nullptr, *uidx = nullptr;
    int *useg = nullptr;        // [group][17] class boundaries of the union
    uint16_t *upos = nullptr;   // [double][string] position in the group's union
    double *c64 = nullptr;
    float *c32 = nullptr;
};
jci_status group_tables_build(const jci_space *s, int spin, GroupTables *t);
void group_tables_free(GroupTables *t);
jci_status group_fill(GroupTables *t, const double *dblH, const float *dblHf, cudaStream_t st);
template <typename T>
jci_status group_launch(const GroupArgs<T> &a, int items, int device, const T *x, T *y,
                        cudaStream_t st);

// Same-spin doubles through (N-2)-electron hole strings, jci_fci_pairs.cu
// (group kernel variants 5 and 6).
struct PairTables {
    int nk = 0, np = 0, NP = 0, nt = 0, ngp = 0, rows = 0;
    std::vector<int> orb;          // the varying orbitals (1-based)
    int *jrow = nullptr;           // [hole string][pair] source string | phase << 31
    uint16_t *gp = nullptr;        // [hole string][pair] orbital pair
    int *pull = nullptr;           // [string][hole] hole string * np + pair
    double *W64 = nullptr;         // [orbital pair][orbital pair]
    float *W32 = nullptr;
    std::vector<double> w64;       // host copies behind the asynchronous uploads
    std::vector<float> w32;
};
jci_status pair_tables_build(const jci_space *s, int spin, PairTables *t);
jci_status pair_fill(const jci_space *s, PairTables *t, cudaStream_t st);
void pair_tables_free(PairTables *t);
size_t pair_smem_bytes(const PairTables &t, int prec);
int pair_block_cols(const PairTables &t, int len, int variant, size_t w);
template <typename T>
jci_status pair_launch(const PairTables &t, int len, int variant, const T *x, T *y, const T *hd,
                       int add, const int *skip, T *E, int device, cudaStream_t st);

// Singles of one spin through (N-1)-electron hole strings, jci_fci_pairs.cu
// (the beta-singles pass of plans 6 and 7 with threads = 0).
struct HsTables {
    int nk = 0, nf = 0, nt = 0, rows = 0;
    int *srow = nullptr;           // [hole string][free orbital] string
    int *sidx = nullptr;           // [hole][x][y] one-body table position | phase << 31, -1 diagonal
    uint16_t *pp = nullptr;        // [hole][x][y] pair | phase << 15
    int *pull = nullptr;           // [string][hole] hole string * nf + free orbital
    double *a1s64 = nullptr;       // [hole][x][y] phase x one-body part
    float *a1s32 = nullptr;
};
jci_status hs_tables_build(const jci_space *s, int spin, HsTables *t);
jci_status hs_fill(HsTables *t, const double *a1T, const float *a1Tf, cudaStream_t st);
void hs_tables_free(HsTables *t);
size_t hs_smem_bytes(int npair, size_t w);
int hs_block_cols(const HsTables &t, int len, size_t w);
template <typename T>
jci_status hs_launch(const HsTables &t, int len, int npair, const T *jc, const T *x, T *y,
                     const int *skip, T *E, int device, cudaStream_t st);

// Generic path (any truncated space), jci_device.cu.
jci_status device_sigma_generic(jci_space *s, int nvec, const void *vin, void *sout,
                                long long ld, int precision, cudaStream_t st);

// Davidson buffers (jci_davidson.cu).
void davidson_free(DeviceState *d);

}  // namespace jci
