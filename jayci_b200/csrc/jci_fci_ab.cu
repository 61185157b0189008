// jci_fci_ab.cu -- the alpha-single x beta-single part of sigma (one-group
// spaces) as one fused kernel: the dense product is computed in column
// chunks that stay in shared memory and are gathered at once.
//
// For one alpha string Ia with alpha singles j -> (Ja_j, phase s_j, pair p_j)
// (hmatels_1x and hmatels_2xab, action_util.c):
//   T[p][Jb] = sum_j s_j (p_j | p) c(Ja_j, Jb)             (rows p < npair)
//   T[U][Jb] = sum_j s_j a1(Ia, j) c(Ja_j, Jb)             (row U = npair)
//   sigma(Ia, Ib) += T[U][Ib] + sum_{m in Ib} T[(mm)][Ib]
//                  + sum_{beta singles Ib -> Jb, pair q, phase t} t T[q][Jb].
// The product chunk T[:, c0 : c0 + CW] is formed in shared memory; every
// term of the sum above whose column Jb (or Ib for the first two) falls in
// the chunk is an entry of a per-chunk list sorted by the string Ib, and the
// thread that owns Ib adds its entries in list order.  Sums are therefore
// taken in one fixed order (chunk, then list) and results are bitwise
// reproducible; T never leaves the SM.
//
// Three product engines:
//  - k_sigma_ab_dmma (FP64, 64-column chunks): the FP64 tensor cores,
//    mma.sync m8n8k4 (tcgen05 has no FP64 kind), with the chunk's entry
//    lists copied into shared memory (cp.async) while the chunk multiplies;
//  - k_sigma_ab_tf32 (FP32, 64-column chunks): the same structure on the
//    TF32 tensor cores with 3xTF32 operand splitting (FP32 accuracy, FP32
//    accumulation);
//  - k_sigma_ab (FP32 and FP64, 32-column chunks): register tiles on the
//    CUDA-core FMA pipes, entry lists read from L2.
#include <cuda_pipeline.h>

#include <algorithm>
#include <vector>

#include "jci_internal.h"
#include "jci_kernels.cuh"

namespace jci {

namespace {

constexpr int kAbThreads = 256;

template <typename T>
__device__ __forceinline__ T ab_flip(T w, uint32_t neg) {
    return neg ? -w : w;
}

__device__ __forceinline__ void ab_dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// ---- CUDA-core engine -------------------------------------------------------
//
// TX threads across the chunk's columns (4 consecutive columns each, so
// CW = 4 TX), TY = 256 / TX threads across the product rows (TM rows each);
// ITEMS beta strings per thread in the gather.  A thread's TM rows of A
// are stored padded to TMP (a multiple of 16 bytes), so per k step it
// reads its A values and its four B values with 16-byte loads.
template <typename T>
struct AbVec;
template <>
struct AbVec<double> {
    using type = double2;
};
template <>
struct AbVec<float> {
    using type = float4;
};

__host__ __device__ constexpr int ab_tmp(int tm, int w) {
    return (tm + 16 / w - 1) / (16 / w) * (16 / w);
}

template <typename T, int TX, int TM, int ITEMS>
__global__ void __launch_bounds__(kAbThreads)
    k_sigma_ab(AbArgs<T> a, const T *__restrict__ V, T *__restrict__ S) {
    if (a.skip && *a.skip) return;
    using VT = typename AbVec<T>::type;
    constexpr int E = 16 / (int)sizeof(T);  // values per 16-byte load
    constexpr int TMP = ab_tmp(TM, (int)sizeof(T));
    constexpr int TY = kAbThreads / TX, CW = 4 * TX, MP = TY * TMP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = a.sa, nb = a.nb;
    T *As = reinterpret_cast<T *>(smem_raw);                        // [K][TY][TMP]
    T *Bs = As + (size_t)K * MP;                                    // [2][K][CW]
    T *Ts = Bs + 2 * (size_t)K * CW;                                // [mrows][CW]
    int *jl = reinterpret_cast<int *>(Ts + (size_t)a.mrows * CW);  // [K]
    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    // B chunks (the alpha-single rows of C, CW columns) are double-buffered:
    // chunk c+1 is copied (cp.async) while chunk c is multiplied
    auto stage = [&](int c, T *buf) {
        const int c0 = c * CW;
        for (int idx = tid; idx < K * CW; idx += kAbThreads) {
            const int j = idx / CW, col = c0 + idx % CW;
            if (col < nb)
                __pipeline_memcpy_async(buf + idx, V + (long long)jl[j] * nb + col, sizeof(T));
            else
                buf[idx] = T(0);
        }
        __pipeline_commit();
    };
    for (int Ia = blockIdx.x; Ia < a.na; Ia += gridDim.x) {
        __syncthreads();
        for (int idx = tid; idx < K * MP; idx += kAbThreads) {
            const int j = idx / MP, pos = idx - j * MP, i = pos % TMP;
            const int m = i < TM ? (pos / TMP) * TM + i : a.mrows;  // padding: zero
            const long long o = (long long)j * a.na + Ia;
            const uint32_t e = a.fsA[o];
            T v = T(0);
            if (m < a.npair) v = a.m2[eri_index(a.fpA[o], m)];
            else if (m == a.npair) v = a.a1A[o];
            As[idx] = ab_flip(v, e >> 31);
            if (pos == 0) jl[j] = (int)(e & 0x3fffffffu);
        }
        T x[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) x[i] = T(0);
        __syncthreads();
        stage(0, Bs);
        for (int ci = 0; ci < a.nchunk; ci++) {
            T *Bc = Bs + (size_t)(ci & 1) * K * CW;
            if (ci + 1 < a.nchunk) {
                stage(ci + 1, Bs + (size_t)((ci + 1) & 1) * K * CW);
                __pipeline_wait_prior(1);
            } else {
                __pipeline_wait_prior(0);
            }
            // also orders the previous chunk's gather before Ts is rewritten
            __syncthreads();
            T acc[TM][4];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[i][q] = T(0);
#pragma unroll 4
            for (int k = 0; k < K; k++) {
                // columns 4 tx .. 4 tx + 3 and the thread's A rows, 16 bytes a load
                T bv[4], av[TMP];
                const VT *br = reinterpret_cast<const VT *>(Bc + k * CW + 4 * tx);
#pragma unroll
                for (int q = 0; q < 4 / E; q++) *reinterpret_cast<VT *>(bv + q * E) = br[q];
                const VT *ar = reinterpret_cast<const VT *>(As + k * MP + ty * TMP);
#pragma unroll
                for (int q = 0; q < TMP / E; q++) *reinterpret_cast<VT *>(av + q * E) = ar[q];
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[i][q] = fma(av[i], bv[q], acc[i][q]);
            }
#pragma unroll
            for (int i = 0; i < TM; i++) {
                const int m = ty * TM + i;
                if (m < a.mrows) {
                    T *dst = Ts + (size_t)m * CW + 4 * tx;
#pragma unroll
                    for (int q = 0; q < 4; q++) dst[q] = acc[i][q];
                }
            }
            __syncthreads();
            // gather: string Ib = tid + 256 i adds its entries of this chunk
            const uint16_t *off = a.off + (size_t)ci * a.offs;
            const uint32_t *ent = a.ent + a.base[ci];
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const int Ib = tid + kAbThreads * i;
                if (Ib < nb) {
                    const int k1 = off[Ib + 1];
                    T s = x[i];
                    for (int k = off[Ib]; k < k1; k++) {
                        const uint32_t e = ent[k];
                        s += ab_flip(Ts[(size_t)((e >> 8) & 0xffffu) * CW + (e & 0xffu)], e >> 31);
                    }
                    x[i] = s;
                }
            }
        }
        T *srow = S + (long long)Ia * nb;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const int Ib = tid + kAbThreads * i;
            if (Ib < nb) srow[Ib] += x[i];
        }
    }
}

// ---- FP64 tensor-core engine ------------------------------------------------
//
// 64-column chunks, eight warps as 2 (rows) x 4 (columns): warp (wm, wn) owns
// the 8x8 tiles of rows 8 (wm MTW + i) (i < MTW) and columns 16 wn + 8 j
// (j < 2).  Per 4-wide k step it loads MTW A fragments and two B fragments
// from shared memory and issues 2 MTW mma.sync.m8n8k4.f64.  Row strides
// are padded to 4 mod 16 doubles (kDmCWP for B, dm_kp for A), so the eight
// quarter-warp fragment loads hit distinct banks.
constexpr int kDmCW = 64, kDmCWP = 68;

__host__ __device__ inline int dm_k4(int K) { return (K + 3) & ~3; }
__host__ __device__ inline int dm_kp(int K) {
    const int k4 = dm_k4(K);
    return k4 + (20 - k4 % 16) % 16;
}

template <int MTW, int ITEMS, int NB>
__global__ void __launch_bounds__(kAbThreads, NB == 1 ? 2 : 1)  // one B buffer: two CTAs per SM
    k_sigma_ab_dmma(AbArgs<double> a, const double *__restrict__ V, double *__restrict__ S) {
    if (a.skip && *a.skip) return;
    constexpr int R8 = 16 * MTW;  // product rows covered (>= mrows)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = a.sa, K4 = dm_k4(K), KP = dm_kp(K), nb = a.nb;
    double *As = reinterpret_cast<double *>(smem_raw);             // [R8][KP]
    double *Bs = As + (size_t)R8 * KP;                             // [NB][K4][kDmCWP]
    double *Ts = Bs + NB * (size_t)K4 * kDmCWP;                    // [mrows][kDmCW]
    uint32_t *es = reinterpret_cast<uint32_t *>(Ts + (size_t)a.mrows * kDmCW);  // [maxent]
    uint16_t *os = reinterpret_cast<uint16_t *>(es + a.maxent);   // [offs]
    int *jl = reinterpret_cast<int *>(os + a.offs);                // [K]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3, wn = warp & 3, wm = warp >> 2;
    // the k rows K..K4-1 of the B buffers stay zero (never staged)
    for (int idx = tid; idx < NB * (K4 - K) * kDmCWP; idx += kAbThreads) {
        const int b = idx / ((K4 - K) * kDmCWP), r = idx % ((K4 - K) * kDmCWP);
        Bs[(size_t)b * K4 * kDmCWP + (size_t)K * kDmCWP + r] = 0.0;
    }
    auto stage_b = [&](int c, double *buf) {
        const int c0 = c * kDmCW;
        if (a.vec) {  // nb even and C 16-byte aligned: column pairs
            for (int idx = tid; idx < K * (kDmCW / 2); idx += kAbThreads) {
                const int j = idx / (kDmCW / 2), cc = 2 * (idx % (kDmCW / 2)), col = c0 + cc;
                double *dst = buf + (size_t)j * kDmCWP + cc;
                if (col < nb)
                    __pipeline_memcpy_async(dst, V + (long long)jl[j] * nb + col, 16);
                else
                    dst[0] = dst[1] = 0.0;
            }
        } else {
            for (int idx = tid; idx < K * kDmCW; idx += kAbThreads) {
                const int j = idx / kDmCW, cc = idx % kDmCW, col = c0 + cc;
                double *dst = buf + (size_t)j * kDmCWP + cc;
                if (col < nb)
                    __pipeline_memcpy_async(dst, V + (long long)jl[j] * nb + col, 8);
                else
                    dst[0] = 0.0;
            }
        }
        __pipeline_commit();
    };
    // the chunk's offsets and entries (rows padded to 16 bytes on the host)
    auto stage_l = [&](int c) {
        const uint16_t *og = a.off + (size_t)c * a.offs;
        for (int idx = tid; idx < a.offs / 8; idx += kAbThreads)
            __pipeline_memcpy_async(os + 8 * idx, og + 8 * idx, 16);
        const uint32_t b0 = a.base[c], n4 = (a.base[c + 1] - b0) / 4;
        for (uint32_t idx = tid; idx < n4; idx += kAbThreads)
            __pipeline_memcpy_async(es + 4 * idx, a.ent + b0 + 4 * idx, 16);
        __pipeline_commit();
    };
    for (int Ia = blockIdx.x; Ia < a.na; Ia += gridDim.x) {
        __syncthreads();
        // A[m][k] = s_k (p_k | m) for m < npair, s_k a1_k for m = npair, 0 beyond
        for (int idx = tid; idx < R8 * K4; idx += kAbThreads) {
            const int m = idx / K4, j = idx - m * K4;
            double v = 0.0;
            if (j < K && m <= a.npair) {
                const long long o = (long long)j * a.na + Ia;
                v = m < a.npair ? a.m2[eri_index(a.fpA[o], m)] : a.a1A[o];
                if (a.fsA[o] >> 31) v = -v;
            }
            As[(size_t)m * KP + j] = v;
        }
        for (int j = tid; j < K; j += kAbThreads)
            jl[j] = (int)(a.fsA[(long long)j * a.na + Ia] & 0x3fffffffu);
        double x[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) x[i] = 0.0;
        __syncthreads();
        stage_b(0, Bs);
        for (int ci = 0; ci < a.nchunk; ci++) {
            const double *Bc = Bs + (size_t)(ci % NB) * K4 * kDmCWP;
            // B chunk ci landed; every thread is past the previous gather, so
            // the lists (and, double-buffered, the other B buffer) may be
            // overwritten
            __pipeline_wait_prior(0);
            __syncthreads();
            stage_l(ci);
            const bool more = ci + 1 < a.nchunk;
            if (NB == 2 && more) stage_b(ci + 1, Bs + (size_t)((ci + 1) & 1) * K4 * kDmCWP);
            double acc[MTW][2][2];
#pragma unroll
            for (int i = 0; i < MTW; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
            const double *ap = As + (size_t)(8 * wm * MTW + g) * KP + t;
            const double *bp = Bc + (size_t)t * kDmCWP + 16 * wn + g;
#pragma unroll 2
            for (int k0 = 0; k0 < K4; k0 += 4) {
                const double b0 = bp[(size_t)k0 * kDmCWP], b1 = bp[(size_t)k0 * kDmCWP + 8];
#pragma unroll
                for (int i = 0; i < MTW; i++) {
                    const double av = ap[(size_t)8 * i * KP + k0];
                    ab_dmma(acc[i][0], av, b0);
                    ab_dmma(acc[i][1], av, b1);
                }
            }
            // fragments: lane holds row g, columns 2t and 2t+1 of each tile
#pragma unroll
            for (int i = 0; i < MTW; i++) {
                const int m = 8 * (wm * MTW + i) + g;
                if (m < a.mrows) {
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        double *dst = Ts + (size_t)m * kDmCW + 16 * wn + 8 * j + 2 * t;
                        dst[0] = acc[i][j][0];
                        dst[1] = acc[i][j][1];
                    }
                }
            }
            if (NB == 2 && more)
                __pipeline_wait_prior(1);  // the lists (B chunk ci+1 may still fly)
            else
                __pipeline_wait_prior(0);
            __syncthreads();
            // single-buffered: chunk ci+1 is copied while chunk ci gathers
            if (NB == 1 && more) stage_b(ci + 1, Bs);
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const int Ib = tid + kAbThreads * i;
                if (Ib < nb) {
                    const int k1 = os[Ib + 1];
                    double s = x[i];
                    for (int k = os[Ib]; k < k1; k++) {
                        const uint32_t e = es[k];
                        const double v = Ts[(size_t)((e >> 8) & 0xffffu) * kDmCW + (e & 0xffu)];
                        s += e >> 31 ? -v : v;
                    }
                    x[i] = s;
                }
            }
        }
        double *srow = S + (long long)Ia * nb;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const int Ib = tid + kAbThreads * i;
            if (Ib < nb) srow[Ib] += x[i];
        }
    }
}

// ---- FP32 tensor-core engine: 3xTF32 -----------------------------------------
//
// The FP32 product on the tensor cores with FP32 accuracy: each FP32
// operand x is split into a TF32 part x_h = tf32(x) and a TF32 remainder
// x_l = tf32(x - x_h), and every 16x8x8 tile takes three mma.sync.m16n8k8
// with FP32 accumulation, a_l b_h + a_h b_l + a_h b_h (the a_l b_l term is
// below FP32 rounding).  64-column chunks; eight warps as 2 (rows) x 4
// (columns): warp (wm, wn) owns the 16x8 tiles of rows 16 (wm MT + i) (i <
// MT) and columns 16 wn + 8 j (j < 2).  Row strides are padded (4 mod 32
// words for A, 8 mod 32 for B) so the fragment loads hit distinct banks.
// Chunk lists, gather and buffering as in k_sigma_ab_dmma.
constexpr int kTfCW = 64, kTfCWP = 72;

__host__ __device__ inline int tf_k8(int K) { return (K + 7) & ~7; }
__host__ __device__ inline int tf_kp(int K) {
    const int k8 = tf_k8(K);
    return k8 + (36 - k8 % 32) % 32;
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// AS = 1: the A panel is split once per alpha string and kept as its TF32
// parts (two panels); AS = 0: A is kept in FP32 and split at every load.
template <int MT, int ITEMS, int NB, int AS>
__global__ void __launch_bounds__(kAbThreads, NB == 1 ? 2 : 1)  // one B buffer: two CTAs per SM
    k_sigma_ab_tf32(AbArgs<float> a, const float *__restrict__ V, float *__restrict__ S) {
    if (a.skip && *a.skip) return;
    constexpr int R16 = 32 * MT;  // product rows covered (>= mrows)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = a.sa, K8 = tf_k8(K), KP = tf_kp(K), nb = a.nb;
    float *As = reinterpret_cast<float *>(smem_raw);               // [1 + AS][R16][KP]
    uint32_t *Ah = reinterpret_cast<uint32_t *>(As);               // AS: TF32 high parts
    uint32_t *Al = Ah + (size_t)R16 * KP;                          // AS: TF32 remainders
    float *Bs = As + (size_t)(1 + AS) * R16 * KP;                  // [NB][K8][kTfCWP]
    float *Ts = Bs + NB * (size_t)K8 * kTfCWP;                     // [mrows][kTfCW]
    uint32_t *es = reinterpret_cast<uint32_t *>(Ts + (size_t)a.mrows * kTfCW);  // [maxent]
    uint16_t *os = reinterpret_cast<uint16_t *>(es + a.maxent);   // [offs]
    int *jl = reinterpret_cast<int *>(os + a.offs);                // [K]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3, wn = warp & 3, wm = warp >> 2;
    // the k rows K..K8-1 of the B buffers stay zero (never staged)
    for (int idx = tid; idx < NB * (K8 - K) * kTfCWP; idx += kAbThreads) {
        const int b = idx / ((K8 - K) * kTfCWP), r = idx % ((K8 - K) * kTfCWP);
        Bs[(size_t)b * K8 * kTfCWP + (size_t)K * kTfCWP + r] = 0.f;
    }
    auto stage_b = [&](int c, float *buf) {
        const int c0 = c * kTfCW;
        if (a.vec) {  // nb a multiple of 4 and C 16-byte aligned: column quads
            for (int idx = tid; idx < K * (kTfCW / 4); idx += kAbThreads) {
                const int j = idx / (kTfCW / 4), cc = 4 * (idx % (kTfCW / 4)), col = c0 + cc;
                float *dst = buf + (size_t)j * kTfCWP + cc;
                if (col < nb)
                    __pipeline_memcpy_async(dst, V + (long long)jl[j] * nb + col, 16);
                else
                    dst[0] = dst[1] = dst[2] = dst[3] = 0.f;
            }
        } else {
            for (int idx = tid; idx < K * kTfCW; idx += kAbThreads) {
                const int j = idx / kTfCW, cc = idx % kTfCW, col = c0 + cc;
                float *dst = buf + (size_t)j * kTfCWP + cc;
                if (col < nb)
                    __pipeline_memcpy_async(dst, V + (long long)jl[j] * nb + col, 4);
                else
                    dst[0] = 0.f;
            }
        }
        __pipeline_commit();
    };
    auto stage_l = [&](int c) {
        const uint16_t *og = a.off + (size_t)c * a.offs;
        for (int idx = tid; idx < a.offs / 8; idx += kAbThreads)
            __pipeline_memcpy_async(os + 8 * idx, og + 8 * idx, 16);
        const uint32_t b0 = a.base[c], n4 = (a.base[c + 1] - b0) / 4;
        for (uint32_t idx = tid; idx < n4; idx += kAbThreads)
            __pipeline_memcpy_async(es + 4 * idx, a.ent + b0 + 4 * idx, 16);
        __pipeline_commit();
    };
    for (int Ia = blockIdx.x; Ia < a.na; Ia += gridDim.x) {
        __syncthreads();
        for (int idx = tid; idx < R16 * K8; idx += kAbThreads) {
            const int m = idx / K8, j = idx - m * K8;
            float v = 0.f;
            if (j < K && m <= a.npair) {
                const long long o = (long long)j * a.na + Ia;
                v = m < a.npair ? a.m2[eri_index(a.fpA[o], m)] : a.a1A[o];
                if (a.fsA[o] >> 31) v = -v;
            }
            if (AS)
                split_tf32(v, Ah[(size_t)m * KP + j], Al[(size_t)m * KP + j]);
            else
                As[(size_t)m * KP + j] = v;
        }
        for (int j = tid; j < K; j += kAbThreads)
            jl[j] = (int)(a.fsA[(long long)j * a.na + Ia] & 0x3fffffffu);
        float x[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) x[i] = 0.f;
        __syncthreads();
        stage_b(0, Bs);
        for (int ci = 0; ci < a.nchunk; ci++) {
            const float *Bc = Bs + (size_t)(ci % NB) * K8 * kTfCWP;
            __pipeline_wait_prior(0);
            __syncthreads();
            stage_l(ci);
            const bool more = ci + 1 < a.nchunk;
            if (NB == 2 && more) stage_b(ci + 1, Bs + (size_t)((ci + 1) & 1) * K8 * kTfCWP);
            float acc[MT][2][4];
#pragma unroll
            for (int i = 0; i < MT; i++)
#pragma unroll
                for (int j = 0; j < 2; j++)
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[i][j][q] = 0.f;
            const float *bp = Bc + (size_t)t * kTfCWP + 16 * wn + g;
#pragma unroll 2
            for (int k0 = 0; k0 < K8; k0 += 8) {
                uint32_t bh[2][2], bl[2][2];
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    split_tf32(bp[(size_t)k0 * kTfCWP + 8 * j], bh[j][0], bl[j][0]);
                    split_tf32(bp[(size_t)(k0 + 4) * kTfCWP + 8 * j], bh[j][1], bl[j][1]);
                }
#pragma unroll
                for (int i = 0; i < MT; i++) {
                    const size_t ao = (size_t)(16 * (wm * MT + i) + g) * KP + t + k0;
                    const size_t off[4] = {0, (size_t)8 * KP, 4, (size_t)8 * KP + 4};
                    uint32_t ah[4], al[4];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        if (AS) {
                            ah[q] = Ah[ao + off[q]];
                            al[q] = Al[ao + off[q]];
                        } else {
                            split_tf32(As[ao + off[q]], ah[q], al[q]);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 2; j++) {
                        mma_tf32(acc[i][j], al, bh[j][0], bh[j][1]);
                        mma_tf32(acc[i][j], ah, bl[j][0], bl[j][1]);
                        mma_tf32(acc[i][j], ah, bh[j][0], bh[j][1]);
                    }
                }
            }
            // fragments: lane holds rows g and g+8, columns 2t and 2t+1 of each tile
#pragma unroll
            for (int i = 0; i < MT; i++) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int m = 16 * (wm * MT + i) + g + 8 * h;
                    if (m < a.mrows) {
#pragma unroll
                        for (int j = 0; j < 2; j++) {
                            float *dst = Ts + (size_t)m * kTfCW + 16 * wn + 8 * j + 2 * t;
                            dst[0] = acc[i][j][2 * h];
                            dst[1] = acc[i][j][2 * h + 1];
                        }
                    }
                }
            }
            if (NB == 2 && more)
                __pipeline_wait_prior(1);  // the lists (B chunk ci+1 may still fly)
            else
                __pipeline_wait_prior(0);
            __syncthreads();
            // single-buffered: chunk ci+1 is copied while chunk ci gathers
            if (NB == 1 && more) stage_b(ci + 1, Bs);
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const int Ib = tid + kAbThreads * i;
                if (Ib < nb) {
                    const int k1 = os[Ib + 1];
                    float sacc = x[i];
                    for (int k = os[Ib]; k < k1; k++) {
                        const uint32_t e = es[k];
                        const float v = Ts[(size_t)((e >> 8) & 0xffffu) * kTfCW + (e & 0xffu)];
                        sacc += e >> 31 ? -v : v;
                    }
                    x[i] = sacc;
                }
            }
        }
        float *srow = S + (long long)Ia * nb;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const int Ib = tid + kAbThreads * i;
            if (Ib < nb) srow[Ib] += x[i];
        }
    }
}

template <typename T>
using AbKernel = void (*)(AbArgs<T>, const T *, T *);

template <typename T, int TX, int ITEMS>
AbKernel<T> ab_kernel_tm(int tm) {
    switch (tm) {
        case 1: return k_sigma_ab<T, TX, 1, ITEMS>;
        case 2: return k_sigma_ab<T, TX, 2, ITEMS>;
        case 3: return k_sigma_ab<T, TX, 3, ITEMS>;
        case 4: return k_sigma_ab<T, TX, 4, ITEMS>;
        case 5: return k_sigma_ab<T, TX, 5, ITEMS>;
        default: break;
    }
    if constexpr (TX == 16) {
        switch (tm) {
            case 6: return k_sigma_ab<T, TX, 6, ITEMS>;
            case 7: return k_sigma_ab<T, TX, 7, ITEMS>;
            case 8: return k_sigma_ab<T, TX, 8, ITEMS>;
            case 9: return k_sigma_ab<T, TX, 9, ITEMS>;
            default: break;
        }
    }
    return nullptr;
}

template <int ITEMS, int NB>
AbKernel<double> dmma_kernel_mt(int mtw) {
    switch (mtw) {
        case 1: return k_sigma_ab_dmma<1, ITEMS, NB>;
        case 2: return k_sigma_ab_dmma<2, ITEMS, NB>;
        case 3: return k_sigma_ab_dmma<3, ITEMS, NB>;
        case 4: return k_sigma_ab_dmma<4, ITEMS, NB>;
        case 5: return k_sigma_ab_dmma<5, ITEMS, NB>;
        case 6: return k_sigma_ab_dmma<6, ITEMS, NB>;
        case 7: return k_sigma_ab_dmma<7, ITEMS, NB>;
        case 8: return k_sigma_ab_dmma<8, ITEMS, NB>;
        case 9: return k_sigma_ab_dmma<9, ITEMS, NB>;
        default: return nullptr;
    }
}

template <int ITEMS, int NB, int AS>
AbKernel<float> tf32_kernel_mt(int mt) {
    switch (mt) {
        case 1: return k_sigma_ab_tf32<1, ITEMS, NB, AS>;
        case 2: return k_sigma_ab_tf32<2, ITEMS, NB, AS>;
        case 3: return k_sigma_ab_tf32<3, ITEMS, NB, AS>;
        case 4: return k_sigma_ab_tf32<4, ITEMS, NB, AS>;
        case 5: return k_sigma_ab_tf32<5, ITEMS, NB, AS>;
        default: return nullptr;
    }
}

// 16-row tiles per warp of the TF32 engine (two warp rows)
int tf_mt(int mrows) { return ((mrows + 15) / 16 + 1) / 2; }

int ab_items(int nb) {
    const int it = (nb + kAbThreads - 1) / kAbThreads;
    return it <= 4 ? 4 : it <= 16 ? 16 : 0;
}

int ab_tm(int mrows, int tx) { return (mrows + kAbThreads / tx - 1) / (kAbThreads / tx); }

// m tiles per warp of the tensor-core engine (two warp rows of 8-row tiles)
int dm_mtw(int mrows) { return ((mrows + 7) / 8 + 1) / 2; }

// The tensor-core engine runs FP64 chunks of 64 columns (tx = 16).
bool use_dmma(int tx, size_t w) { return tx == 16 && w == sizeof(double); }
// In FP32, 64-column chunks (tx = 16) run 3xTF32 on the tensor cores.
bool use_tf32(int tx, size_t w) { return tx == 16 && w == sizeof(float); }

template <typename T>
AbKernel<T> ab_kernel(int tx, int mrows, int items, int nbuf) {
    if constexpr (sizeof(T) == sizeof(float)) {
        if (use_tf32(tx, sizeof(T))) {
            // variant 3: one B buffer and the A panel pre-split; 1: one B
            // buffer; 2: two B buffers
            const int mt = tf_mt(mrows);
            if (nbuf == 3)
                return items == 4 ? tf32_kernel_mt<4, 1, 1>(mt) : tf32_kernel_mt<16, 1, 1>(mt);
            if (nbuf == 1)
                return items == 4 ? tf32_kernel_mt<4, 1, 0>(mt) : tf32_kernel_mt<16, 1, 0>(mt);
            return items == 4 ? tf32_kernel_mt<4, 2, 0>(mt) : tf32_kernel_mt<16, 2, 0>(mt);
        }
    }
    if constexpr (sizeof(T) == sizeof(double)) {
        if (use_dmma(tx, sizeof(T))) {
            const int mtw = dm_mtw(mrows);
            if (nbuf == 1)
                return items == 4 ? dmma_kernel_mt<4, 1>(mtw) : dmma_kernel_mt<16, 1>(mtw);
            return items == 4 ? dmma_kernel_mt<4, 2>(mtw) : dmma_kernel_mt<16, 2>(mtw);
        }
    }
    const int tm = ab_tm(mrows, tx);
    if (tx == 8) return items == 4 ? ab_kernel_tm<T, 8, 4>(tm) : ab_kernel_tm<T, 8, 16>(tm);
    if (tx == 16) return items == 4 ? ab_kernel_tm<T, 16, 4>(tm) : ab_kernel_tm<T, 16, 16>(tm);
    return nullptr;
}

// Row stride of the offsets (nb + 1 rounded up to 8: 16-byte rows) and the
// longest chunk list: every beta string is the target of exactly sb singles
// in a one-group space, so a full chunk holds cw (1 + nelb + sb) entries,
// rounded up to 4 (16-byte lists).
int ab_offs(int nb) { return (nb + 1 + 7) / 8 * 8; }
int ab_maxent(const AbShape &sh, int cw) { return (cw * (1 + sh.nelb + sh.sb) + 3) / 4 * 4; }

}  // namespace

// Dynamic shared memory of each engine; nbuf: B buffers of the tensor-core
// engine; maxent, offs: longest chunk list and offset row stride.
static size_t ab_smem_bytes(int tx, size_t w, int sa, int mrows, int nbuf, int maxent, int offs) {
    if (use_tf32(tx, w)) {
        // nbuf: the variant (3: one B buffer, A pre-split; 1: one B buffer; 2: two)
        const int K8 = tf_k8(sa), KP = tf_kp(sa), R16 = 32 * tf_mt(mrows);
        const int apanels = nbuf == 3 ? 2 : 1, bbufs = nbuf == 2 ? 2 : 1;
        return ((size_t)apanels * R16 * KP + (size_t)bbufs * K8 * kTfCWP +
                (size_t)mrows * kTfCW) * w +
               (size_t)maxent * 4 + (size_t)offs * 2 + (size_t)sa * 4 + 16;
    }
    if (use_dmma(tx, w)) {
        const int K4 = dm_k4(sa), KP = dm_kp(sa), R8 = 16 * dm_mtw(mrows);
        return ((size_t)R8 * KP + (size_t)nbuf * K4 * kDmCWP + (size_t)mrows * kDmCW) * w +
               (size_t)maxent * 4 + (size_t)offs * 2 + (size_t)sa * 4 + 16;
    }
    const int cw = 4 * tx, mp = (kAbThreads / tx) * ab_tmp(ab_tm(mrows, tx), (int)w);
    return ((size_t)sa * mp + 2 * (size_t)sa * cw + (size_t)mrows * cw) * w + (size_t)sa * 4 + 16;
}

size_t ab_smem(const AbShape &sh, int tx, size_t w) {
    return ab_smem_bytes(tx, w, sh.sa, sh.npair + 1, 2, ab_maxent(sh, 4 * tx), ab_offs(sh.nb));
}

bool ab_possible(const AbShape &sh, int tx, size_t w, size_t smem_max) {
    const int mrows = sh.npair + 1;
    if (tx != 8 && tx != 16) return false;
    if (!ab_items(sh.nb) || sh.sa < 1 || mrows > 65535) return false;
    if (use_tf32(tx, w)) {
        if (tf_mt(mrows) > 5) return false;
    } else if (use_dmma(tx, w)) {
        if (dm_mtw(mrows) > 9) return false;
    } else if (ab_tm(mrows, tx) > (tx == 16 ? 9 : 5)) {
        return false;
    }
    return ab_smem(sh, tx, w) <= smem_max;
}

// Per-chunk entry lists of the beta side (see the header comment): for
// chunk c (columns [c cw, (c+1) cw)) and string Ib, entries
// off[c][Ib] .. off[c][Ib+1] - 1 of the chunk's list starting at base[c];
// an entry is col | row << 8 | phase << 31 with row the product row (pair,
// or npair for the one-body row).  Order within (c, Ib): the one-body row,
// the Coulomb rows (mm) in string order, then the singles in list order.
// Offset rows are padded to 8 entries and lists to 4 (16-byte copies).
jci_status ab_tables_build(const jci_space *s, int npair, int tx, AbTables *t) {
    const SpinSpace &B = s->sp[1];
    const int nb = B.nstr, cw = 4 * tx, nchunk = (nb + cw - 1) / cw, offs = ab_offs(nb);
    if (nb < 1 || npair + 1 > 65535) return JCI_ERR_SPACE;
    auto each = [&](auto fn) {
        for (int i = 0; i < nb; i++) {
            const uint32_t c = (uint32_t)(i / cw), col = (uint32_t)(i % cw);
            fn(c, i, col | ((uint32_t)npair << 8));
            for (int e = 0; e < B.nelec; e++) {
                const int m = B.istr[(size_t)i * B.nelec + e];
                fn(c, i, col | ((uint32_t)pair_index(m, m) << 8));
            }
            for (long long k = B.soff[i]; k < B.soff[i + 1]; k++) {
                const Exc &x = B.sing[k];
                fn((uint32_t)(x.target / cw), i,
                   (uint32_t)(x.target % cw) | ((uint32_t)pair_index(x.io0, x.fo0) << 8) |
                       (x.sign < 0 ? 0x80000000u : 0u));
            }
        }
    };
    std::vector<uint32_t> cnt((size_t)nchunk * nb, 0);
    each([&](uint32_t c, int i, uint32_t) { cnt[(size_t)c * nb + i]++; });
    std::vector<uint16_t> off((size_t)nchunk * offs, 0);
    std::vector<uint32_t> base(nchunk + 1, 0);
    uint32_t maxent = 4;
    for (int c = 0; c < nchunk; c++) {
        uint32_t run = 0;
        for (int i = 0; i < nb; i++) {
            off[(size_t)c * offs + i] = (uint16_t)run;
            run += cnt[(size_t)c * nb + i];
            if (run > 65535) return JCI_ERR_SPACE;
        }
        for (int i = nb; i < offs; i++) off[(size_t)c * offs + i] = (uint16_t)run;
        const uint32_t padded = (run + 3) / 4 * 4;
        maxent = std::max(maxent, padded);
        base[c + 1] = base[c] + padded;
    }
    std::vector<uint32_t> ent(std::max<uint32_t>(base[nchunk], 4), 0);
    std::vector<uint32_t> pos(cnt.size());
    for (int c = 0; c < nchunk; c++)
        for (int i = 0; i < nb; i++) pos[(size_t)c * nb + i] = base[c] + off[(size_t)c * offs + i];
    each([&](uint32_t c, int i, uint32_t e) { ent[pos[(size_t)c * nb + i]++] = e; });
    AbTables h;
    h.tx = tx;
    h.nchunk = nchunk;
    h.offs = offs;
    h.maxent = (int)maxent;
    jci_status r = JCI_OK;
    if (cudaMalloc(&h.off, off.size() * sizeof(uint16_t)) != cudaSuccess ||
        cudaMalloc(&h.base, base.size() * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&h.ent, ent.size() * sizeof(uint32_t)) != cudaSuccess)
        r = JCI_ERR_CUDA;
    if (!r && (cudaMemcpy(h.off, off.data(), off.size() * sizeof(uint16_t),
                          cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(h.base, base.data(), base.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(h.ent, ent.data(), ent.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice) != cudaSuccess))
        r = JCI_ERR_CUDA;
    if (r) {
        ab_tables_free(&h);
        return r;
    }
    *t = h;
    return JCI_OK;
}

void ab_tables_free(AbTables *t) {
    cudaFree(t->off);
    cudaFree(t->base);
    cudaFree(t->ent);
    *t = AbTables();
}

// Persistent launch: one wave of resident CTAs walks the alpha strings.
// The caller's AbShape-derived limits (ab_possible) must hold, and the
// tables must be those of tx; the smem size uses the tables' longest list.
template <typename T>
jci_status ab_launch(const AbArgs<T> &a, int tx, int device, const T *v, T *o,
                     cudaStream_t st) {
    const int items = ab_items(a.nb);
    if (!items || a.nchunk != (a.nb + 4 * tx - 1) / (4 * tx)) return JCI_ERR_SPACE;
    // The tensor-core engine single-buffers its B chunks when that lets two
    // CTAs share an SM (the other CTA hides the copy); else it double-buffers.
    AbKernel<T> kern = nullptr;
    size_t smem = 0;
    int occ = 0, nsm = 0;
    for (int nbuf : {3, 1, 2}) {
        if (nbuf == 3 && !use_tf32(tx, sizeof(T))) continue;
        if (nbuf == 1 && !use_dmma(tx, sizeof(T)) && !use_tf32(tx, sizeof(T))) continue;
        kern = ab_kernel<T>(tx, a.mrows, items, nbuf);
        if (!kern) return JCI_ERR_SPACE;
        smem = ab_smem_bytes(tx, sizeof(T), a.sa, a.mrows, nbuf, a.maxent, a.offs);
        JCI_CUDA(smem_optin(kern));
        JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kAbThreads, smem));
        if (nbuf == 2 || occ >= 2) break;
    }
    if (occ < 1) return JCI_ERR_SPACE;
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(a.na, nsm * occ));
    kern<<<grid, kAbThreads, smem, st>>>(a, v, o);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

template jci_status ab_launch<double>(const AbArgs<double> &, int, int, const double *, double *,
                                      cudaStream_t);
template jci_status ab_launch<float>(const AbArgs<float> &, int, int, const float *, float *,
                                     cudaStream_t);

}  // namespace jci
