// jci_fci_tc.cu -- the FP32 alpha-single x beta-single part of sigma (one-group
// spaces) on the 5th-generation tensor cores: tcgen05.mma kind::tf32 with the
// product chunk accumulated in tensor memory.
//
// The arithmetic is that of the fused product in jci_fci_ab.cu (hmatels_1x
// and hmatels_2xab, action_util.c:210,250): for one alpha string Ia,
//   T[p][Jb] = sum_j A[p][j] c(Ja_j, Jb),  A[p][j] = s_j (p_j | p)  (p < npair)
//   T[U][Jb] = sum_j s_j a1(Ia, j) c(Ja_j, Jb)                      (row U = npair)
// computed in column chunks of CW beta strings, then gathered over the
// per-chunk entry lists (ab_tables_build) by the thread that owns each beta
// string, in list order, so the sum order is fixed and results are bitwise
// reproducible.
//
// FP32 accuracy from TF32 tensor cores (3xTF32): every operand x is split as
// x_h = tf32(x), x_l = tf32(x - x_h), and each tile takes
// A_l B_h + A_h B_l + A_h B_h with FP32 accumulation in tensor memory.
//
// Per chunk the CTA (512 threads) works as a pipeline over two B buffers and
// two tensor-memory accumulators; in step c:
//   1. all threads split B(c+1) -- rows Ja_j of C, columns of chunk c+1,
//      copied raw one step earlier -- in place into TF32 high and low parts,
//      in the K-major core-matrix layout the MMA reads (8 rows x 16 bytes
//      per core matrix, no swizzle);
//   2. one thread issues the MMAs of chunk c+1 (3 x K8/8 tcgen05.mma of
//      128 x CW x 8 per 128-row tile), committed to an mbarrier, and the
//      bulk copy (cp.async.bulk) of chunk c's entry lists;
//   3. all threads wait for chunk c's MMAs; its B buffer takes the raw copy
//      (cp.async) of B(c+2) at once, and its accumulator moves tensor
//      memory -> registers -> shared memory (tcgen05.ld);
//   4. all threads gather chunk c.
// Chunk c+1's MMAs run under chunk c's extraction and gather, and B(c+2)'s
// copies land under them too.  Every wait is bounded (about one second of global time); on
// expiry the kernel records an error, leaves the remaining work, waits (also
// bounded) for its committed MMAs and releases its tensor memory.
//
// Shared memory (bytes, K8 = alpha singles rounded up to 8, MT 128-row tiles):
//   A_h, A_l  2 x MT x 128 x K8 x 4     B_h, B_l  2 buffers x 2 x CW x K8 x 4
//   T         mrows x (CW + 4) x 4      lists     maxent x 4 + offs x 2
#include <cuda_pipeline.h>

#include <algorithm>
#include <cstdint>

#include "jci_internal.h"
#include "jci_kernels.cuh"

namespace jci {

namespace {


__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t tc_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// K-major operand tile without swizzle: element (row r, k) of a tile with
// K8 columns sits at (r / 8) * SBO + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4
// bytes, SBO = K8 * 32 (the 8-row groups follow each other; within one, the
// K8 / 4 core matrices of 8 rows x 16 bytes follow each other).
__device__ __forceinline__ uint32_t tc_off(int r, int k, int K8) {
    return (uint32_t)((r >> 3) * (K8 * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// Shared-memory matrix descriptor (tcgen05): start address, leading-dimension
// byte offset (K direction, between core matrices), stride-dimension byte
// offset (between 8-row groups), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                       uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase with the given parity of an mbarrier; false after about
// one second of global time (or 2^26 attempts) without completion.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    for (int it = 0; it < (1 << 26); it++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255) == 255 && global_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
        "[%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Tensor-memory columns: two accumulators of MT tiles of CW columns, rounded
// up to a power of two (at least 32).
__host__ __device__ constexpr int tc_cols(int mt, int cw) {
    return 2 * mt * cw <= 32 ? 32 : 2 * mt * cw <= 64 ? 64 : 2 * mt * cw <= 128 ? 128 : 256;
}

struct TcLayout {
    uint32_t ah, al, bh, bl, bstride, ts, es, os, jl, bar, tmem;
    size_t total;
};

__host__ __device__ inline int tc_k8(int K) { return (K + 7) & ~7; }

// Byte offsets of every shared-memory region (16-byte aligned, mbarriers 8).
__host__ __device__ inline TcLayout tc_layout(int K, int mt, int cw, int mrows, int maxent,
                                              int offs) {
    const int K8 = tc_k8(K);
    TcLayout L;
    const uint32_t atile = (uint32_t)(128 * K8 * 4), btile = (uint32_t)(cw * K8 * 4);
    L.ah = 0;
    L.al = L.ah + mt * atile;
    L.bh = L.al + mt * atile;
    L.bl = L.bh + btile;
    L.bstride = 2 * btile;  // buffer b: bh + b * bstride, bl + b * bstride
    L.ts = L.bh + 2 * L.bstride;
    L.es = L.ts + (uint32_t)(((size_t)mrows * (cw + 4) * 4 + 15) / 16 * 16);
    L.os = L.es + (uint32_t)maxent * 4;
    L.jl = L.os + (uint32_t)((offs * 2 + 15) / 16 * 16);
    L.bar = L.jl + (uint32_t)((K * 4 + 15) / 16 * 16);
    L.tmem = L.bar + 3 * 8;
    L.total = L.tmem + 16;
    return L;
}

template <int NT, int CW, int MT, int ITEMS>
__global__ void __launch_bounds__(NT, 1)
    k_sigma_ab_tc(AbArgs<float> a, const float *__restrict__ V, float *__restrict__ S,
                  int *status) {
    if (a.skip && *a.skip) return;
    constexpr int CWP = CW + 4;  // T row stride: rows shift banks by 16 bytes
    constexpr int NCOL = tc_cols(MT, CW);
    extern __shared__ __align__(1024) unsigned char smem[];
    const int K = a.sa, K8 = tc_k8(K), nb = a.nb;
    const TcLayout L = tc_layout(K, MT, CW, a.mrows, a.maxent, a.offs);
    const uint32_t sbase = smem_u32(smem);
    float *Ts = reinterpret_cast<float *>(smem + L.ts);
    const uint32_t *es = reinterpret_cast<const uint32_t *>(smem + L.es);
    const uint16_t *os = reinterpret_cast<const uint16_t *>(smem + L.os);
    int *jl = reinterpret_cast<int *>(smem + L.jl);
    const uint32_t bar_mma0 = sbase + L.bar, bar_list = sbase + L.bar + 16;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.tmem);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile(
            "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                smem_u32(tmem_slot)),
            "r"(NCOL)
            : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar_mma0, 1);
        mbar_init(bar_mma0 + 8, 1);
        mbar_init(bar_list, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    uint32_t ph_mma[2] = {0u, 0u}, ph_list = 0u;
    // thread 0's count of committed MMA groups and bulk list copies not yet
    // waited for (drained before exit after a failed wait)
    int issued[2] = {0, 0}, lists = 0;
    bool failed = false;

    // Raw B chunk c into buffer b: rows Ja_j of C, the chunk's columns, as
    // plain FP32 values at their places in the high-part tile.  A thread
    // copies whole 16-byte pieces -- 4 consecutive k of one column, one
    // 4-byte cp.async each (the 4 values come from 4 rows of C) -- and later
    // splits exactly those pieces, so the split needs only its own copies
    // (no barrier between copy and split).  Rows k >= K and columns past nb
    // are zeros written directly.
    auto fetch_b = [&](int c, int b) {
        const int c0 = c * CW;
        const uint32_t bh = L.bh + (uint32_t)b * L.bstride;
        for (int idx = tid; idx < CW * (K8 / 4); idx += NT) {
            const int n = idx % CW, kq = idx / CW, col = c0 + n;
            float *dst = reinterpret_cast<float *>(smem + bh + tc_off(n, 4 * kq, K8));
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = 4 * kq + u;
                if (k < K && col < nb)
                    __pipeline_memcpy_async(dst + u, V + (long long)jl[k] * nb + col, 4);
                else
                    dst[u] = 0.f;
            }
        }
        __pipeline_commit();
    };
    // Split this thread's pieces of the landed raw chunk in buffer b in
    // place: high part stays, remainder to the low-part tile.
    auto split_b = [&](int b) {
        const uint32_t bh = L.bh + (uint32_t)b * L.bstride, bl = L.bl + (uint32_t)b * L.bstride;
        for (int idx = tid; idx < CW * (K8 / 4); idx += NT) {
            const int n = idx % CW, kq = idx / CW;
            const uint32_t o = tc_off(n, 4 * kq, K8);
            uint4 x = *reinterpret_cast<const uint4 *>(smem + bh + o);
            uint4 hi, lo;
            const uint32_t *xv = &x.x;
            uint32_t *h = &hi.x, *l = &lo.x;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float f = __uint_as_float(xv[u]);
                h[u] = tc_tf32(f);
                l[u] = tc_tf32(f - __uint_as_float(h[u]));
            }
            *reinterpret_cast<uint4 *>(smem + bh + o) = hi;
            *reinterpret_cast<uint4 *>(smem + bl + o) = lo;
        }
    };
    // MMAs of the chunk in buffer b (one thread): per 128-row tile, per
    // 8-wide k step, A_l B_h + A_h B_l + A_h B_h into accumulator b.
    auto issue = [&](int b) {
        tc_fence_after();
        const uint32_t idesc = tc_idesc(CW), sbo = (uint32_t)(K8 * 32);
        const uint32_t bh = sbase + L.bh + (uint32_t)b * L.bstride;
        const uint32_t bl = sbase + L.bl + (uint32_t)b * L.bstride;
#pragma unroll
        for (int t = 0; t < MT; t++) {
            const uint32_t d = tmem + (uint32_t)((b * MT + t) * CW);
            const uint32_t ah = sbase + L.ah + (uint32_t)(t * 128 * K8 * 4);
            const uint32_t al = sbase + L.al + (uint32_t)(t * 128 * K8 * 4);
            for (int s = 0; s < K8 / 8; s++) {
                const uint32_t ko = (uint32_t)(s * 256);
                tc_mma(d, tc_desc(al + ko, 128, sbo), tc_desc(bh + ko, 128, sbo), idesc,
                       s > 0 ? 1u : 0u);
                tc_mma(d, tc_desc(ah + ko, 128, sbo), tc_desc(bl + ko, 128, sbo), idesc, 1u);
                tc_mma(d, tc_desc(ah + ko, 128, sbo), tc_desc(bh + ko, 128, sbo), idesc, 1u);
            }
        }
        tc_commit(bar_mma0 + 8 * b);
    };

    for (int Ia = blockIdx.x; Ia < a.na && !failed; Ia += gridDim.x) {
        // A panel of this alpha string (split) and its single targets
        for (int idx = tid; idx < MT * 128 * (K8 / 4); idx += NT) {
            const int m = idx % (MT * 128), kq = idx / (MT * 128);
            float v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int j = 4 * kq + u;
                v[u] = 0.f;
                if (j < K && m <= a.npair) {
                    const long long o = (long long)j * a.na + Ia;
                    v[u] = m < a.npair ? a.m2[eri_index(a.fpA[o], m)] : a.a1A[o];
                    if (a.fsA[o] >> 31) v[u] = -v[u];
                }
            }
            uint4 hi, lo;
            uint32_t *h = &hi.x, *l = &lo.x;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                h[u] = tc_tf32(v[u]);
                l[u] = tc_tf32(v[u] - __uint_as_float(h[u]));
            }
            const int t = m / 128, r = m % 128;
            const uint32_t o = (uint32_t)(t * 128 * K8 * 4) + tc_off(r, 4 * kq, K8);
            *reinterpret_cast<uint4 *>(smem + L.ah + o) = hi;
            *reinterpret_cast<uint4 *>(smem + L.al + o) = lo;
        }
        for (int j = tid; j < K; j += NT)
            jl[j] = (int)(a.fsA[(long long)j * a.na + Ia] & 0x3fffffffu);
        __syncthreads();  // jl before the B copies read it
        fetch_b(0, 0);
        if (a.nchunk > 1) fetch_b(1, 1);  // the previous string's MMAs are all done
        __pipeline_wait_prior(a.nchunk > 1 ? 1 : 0);  // this thread's raw B(0) pieces
        split_b(0);
        fence_proxy_async();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            issue(0);
            issued[0]++;
        }
        float x[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) x[i] = 0.f;
        for (int ci = 0; ci < a.nchunk; ci++) {
            const int b = ci & 1;
            const bool more = ci + 1 < a.nchunk;
            __pipeline_wait_prior(0);  // this thread's raw B(ci+1) pieces
            if (more) split_b(b ^ 1);
            fence_proxy_async();
            tc_fence_before();
            __syncthreads();  // B(ci+1) split; gather(ci-1) and its T reads done
            if (tid == 0) {
                // the chunk's entry lists, by bulk copy
                const uint32_t e0 = a.base[ci], ne = a.base[ci + 1] - e0;
                mbar_expect_tx(bar_list, ne * 4 + (uint32_t)a.offs * 2);
                bulk_g2s(sbase + L.os, a.off + (size_t)ci * a.offs, (uint32_t)a.offs * 2,
                         bar_list);
                if (ne) bulk_g2s(sbase + L.es, a.ent + e0, ne * 4, bar_list);
                lists++;
                if (more) {
                    issue(b ^ 1);
                    issued[b ^ 1]++;
                }
            }
            // chunk ci's MMAs done: its B buffer takes raw B(ci+2) now, and its
            // accumulator goes to T in shared memory
            bool ok = mbar_wait(bar_mma0 + 8 * b, ph_mma[b]);
            if (ok) {
                ph_mma[b] ^= 1u;
                if (tid == 0) issued[b]--;
            }
            tc_fence_after();
            if (ok && ci + 2 < a.nchunk) fetch_b(ci + 2, b);
            // every warp moves one 8-column slice of one tile: (tile, slice)
            // units of 128 lanes x 8 columns, warp quarter (warp & 3) -> lanes
            const int row = 32 * (warp & 3) + lane;
            if (ok) {
                constexpr int NS = CW / 8;  // slices per tile
                for (int u = warp >> 2; u < MT * NS; u += NT / 128) {
                    const int t = u / NS, c8 = 8 * (u % NS), m = 128 * t + row;
                    uint32_t r[8];
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]),
                          "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                        : "r"(tmem + ((uint32_t)(32 * (warp & 3)) << 16) +
                              (uint32_t)((b * MT + t) * CW + c8))
                        : "memory");
                    tc_wait_ld();
                    if (m < a.mrows) {
                        float4 *dst = reinterpret_cast<float4 *>(Ts + (size_t)m * CWP + c8);
                        dst[0] = make_float4(__uint_as_float(r[0]), __uint_as_float(r[1]),
                                             __uint_as_float(r[2]), __uint_as_float(r[3]));
                        dst[1] = make_float4(__uint_as_float(r[4]), __uint_as_float(r[5]),
                                             __uint_as_float(r[6]), __uint_as_float(r[7]));
                    }
                }
            }
            if (ok && mbar_wait(bar_list, ph_list)) {
                ph_list ^= 1u;
                if (tid == 0) lists--;
            } else {
                ok = false;
            }
            tc_fence_before();
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            // gather: string Ib = tid + NT i adds its entries of this chunk
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const int Ib = tid + NT * i;
                if (Ib < nb) {
                    const int k1 = os[Ib + 1];
                    float s = x[i];
                    for (int k = os[Ib]; k < k1; k++) {
                        const uint32_t e = es[k];
                        const float v = Ts[(size_t)((e >> 8) & 0xffffu) * CWP + (e & 0xffu)];
                        s += e >> 31 ? -v : v;
                    }
                    x[i] = s;
                }
            }
        }
        __pipeline_wait_prior(0);
        if (failed) break;
        float *srow = S + (long long)Ia * nb;
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const int Ib = tid + NT * i;
            if (Ib < nb) srow[Ib] += x[i];
        }
        __syncthreads();  // the A panel and jl are rewritten for the next string
    }
    if (failed) {
        // leave nothing in flight: wait (bounded) for the committed MMA groups
        if (tid == 0) {
            for (int b = 0; b < 2; b++)
                for (; issued[b] > 0 && mbar_wait(bar_mma0 + 8 * b, ph_mma[b]); issued[b]--)
                    ph_mma[b] ^= 1u;
            for (; lists > 0 && mbar_wait(bar_list, ph_list); lists--) ph_list ^= 1u;
            if (status) atomicExch(status, 1);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(NCOL)
                     : "memory");
    }
}

using TcKernel = void (*)(AbArgs<float>, const float *, float *, int *);

// 512 threads per CTA (16 warps hide the copy and gather latency of the one
// CTA an SM holds) and 4, 8, 16 or 32 beta strings per thread, up to 16384
// beta strings -- 32 per thread with 32-column chunks only: the 64-column
// form would exceed the 128 registers a thread of a 512-thread CTA may hold.
constexpr int kTcThreads = 512;

int tc_items(int nb) {
    const int it = (nb + kTcThreads - 1) / kTcThreads;
    return it <= 4 ? 4 : it <= 8 ? 8 : it <= 16 ? 16 : it <= 32 ? 32 : 0;
}

template <int CW, int MT>
TcKernel tc_kernel_items(int items) {
    if (items == 4) return k_sigma_ab_tc<kTcThreads, CW, MT, 4>;
    if (items == 8) return k_sigma_ab_tc<kTcThreads, CW, MT, 8>;
    if (items == 16) return k_sigma_ab_tc<kTcThreads, CW, MT, 16>;
    if constexpr (CW == 32) {
        if (items == 32) return k_sigma_ab_tc<kTcThreads, CW, MT, 32>;
    }
    return nullptr;
}

TcKernel tc_kernel(int cw, int mt, int items) {
    if (cw == 64) return mt == 1 ? tc_kernel_items<64, 1>(items) : tc_kernel_items<64, 2>(items);
    if (cw == 32) return mt == 1 ? tc_kernel_items<32, 1>(items) : tc_kernel_items<32, 2>(items);
    return nullptr;
}

}  // namespace

// Shared memory of the tensor-memory engine for chunk width cw, or 0 when
// the shape is outside its limits (at most 256 product rows, 64 alpha
// singles, 16384 beta strings -- more than 4096 with 32-column chunks only).
size_t tc_smem(const AbShape &sh, int cw) {
    const int mrows = sh.npair + 1, mt = (mrows + 127) / 128;
    if ((cw != 32 && cw != 64) || mt > 2 || sh.sa < 1 || sh.sa > 64 || sh.nb < 1 ||
        !tc_items(sh.nb) || !tc_kernel(cw, mt, tc_items(sh.nb)))
        return 0;
    const int maxent = (cw * (1 + sh.nelb + sh.sb) + 3) / 4 * 4;
    const int offs = (sh.nb + 1 + 7) / 8 * 8;
    return tc_layout(sh.sa, mt, cw, mrows, maxent, offs).total;
}

bool tc_possible(const AbShape &sh, int cw, size_t smem_max) {
    const size_t b = tc_smem(sh, cw);
    return b > 0 && b <= smem_max;
}

// Persistent launch: one CTA per SM walks the alpha strings.  The tables are
// those of the chunk width cw (tx = cw / 4).
jci_status tc_launch(const AbArgs<float> &a, int cw, int device, const float *v, float *o,
                     int *status, cudaStream_t st) {
    const int mt = (a.mrows + 127) / 128, items = tc_items(a.nb);
    TcKernel kern = tc_kernel(cw, mt, items);
    if (!kern || a.nchunk != (a.nb + cw - 1) / cw || a.sa > 64) return JCI_ERR_SPACE;
    const size_t smem = tc_layout(a.sa, mt, cw, a.mrows, a.maxent, a.offs).total;
    const int nt = kTcThreads;
    JCI_CUDA(smem_optin(kern));
    int occ = 0, nsm = 0;
    JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, nt, smem));
    if (occ < 1) return JCI_ERR_SPACE;
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const int grid = std::max(1, std::min(a.na, nsm));
    kern<<<grid, nt, smem, st>>>(a, v, o, status);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

}  // namespace jci
