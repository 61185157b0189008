// jci_fci_group.cu -- same-spin doubles of the one-group sigma as a product
// over groups of consecutive strings (hmatels_2xaa / hmatels_2xbb,
// action_util.c).
//
// For output rows I in a group G of kGroupRows consecutive strings, the
// union U_G of their double-excitation targets is listed once, and
//   Y[I][c] = sum_{J in U_G} H[I][J] X[J][c]   (+ hd[I][c] X[I][c])
// with H[I][J] the double's value with phase, or 0 when I does not reach J.
// Consecutive strings share most targets (16 rows of FCI(14,14) reach 3.7x
// fewer distinct rows than they have doubles), so every source row
// segment is read from L2 once per group instead of once per row.  The
// union is sorted by the set of row quads (rows 4q..4q+3) that reach each
// entry, and each such class runs a loop compiled for its quads, so the
// zero coefficients of the other quads cost neither bytes nor FMAs.  The
// sums run in a fixed order (class, then string), so results are bitwise
// reproducible.
#include <cuda_pipeline.h>

#include <algorithm>
#include <vector>

#include "jci_internal.h"
#include "jci_kernels.cuh"

namespace jci {

namespace {

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
    using type = double2;
};
template <>
struct Vec16<float> {
    using type = float4;
};

constexpr int kGroupChunk = 64;  // union entries per staged chunk

// The entries k0..k1-1 of the staged chunk (coefficient rows cs, source
// rows js) that belong to class QM: reached only by the row quads set in
// QM (bit q: rows 4q..4q+3), so the FMAs of the other quads, whose
// coefficients are all zero, are not issued.  k0 and k1 are multiples of
// 4; the caller takes every STRIDE-th entry quad from k0 (STRIDE 1: all).
template <typename T, int ITEMS, int QM, int STRIDE = 1>
__device__ __forceinline__ void group_class(T (&acc)[kGroupRows][ITEMS],
                                            const T *__restrict__ X,
                                            const T (*__restrict__ cs)[kGroupRows],
                                            const int *__restrict__ js, const int (&col)[ITEMS],
                                            const bool (&in)[ITEMS], int len, int k0, int k1) {
    using V = typename Vec16<T>::type;
    constexpr int E = 16 / (int)sizeof(T);  // rows per 16-byte piece
    constexpr int QE = 4 / E;               // pieces per row quad
    for (int k = k0; k < k1; k += 4 * STRIDE) {
        T x[4][ITEMS];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const T *src = X + (long long)js[k + q] * len;
#pragma unroll
            for (int i = 0; i < ITEMS; i++) x[q][i] = in[i] ? src[col[i]] : T(0);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const V *h = reinterpret_cast<const V *>(cs[k + q]);
#pragma unroll
            for (int qd = 0; qd < 4; qd++) {
                if ((QM >> qd) & 1) {  // a constant once the loop is unrolled
#pragma unroll
                    for (int pe = 0; pe < QE; pe++) {
                        const V hv = h[qd * QE + pe];
                        const T *he = reinterpret_cast<const T *>(&hv);
#pragma unroll
                        for (int e = 0; e < E; e++) {
                            const int r = 4 * qd + pe * E + e;
#pragma unroll
                            for (int i = 0; i < ITEMS; i++)
                                acc[r][i] = fma(he[e], x[q][i], acc[r][i]);
                        }
                    }
                }
            }
        }
    }
}

// Y[I][c] for the kGroupRows rows of group blockIdx.x and the columns
// c0 + tid + NT i (i < ITEMS) of segment blockIdx.y.  The group's union
// entries come sorted by class (the set of row quads that reach them), and
// class QM covers entries useg[g][QM] .. useg[g][QM + 1] - 1; chunks of
// kGroupChunk entries are staged in shared memory (cp.async, double-
// buffered) and each class's part of a chunk runs its own loop.
template <typename T, int NT, int ITEMS>
__global__ void __launch_bounds__(NT, 512 / NT)  // at least 16 warps per SM
    k_sigma_group(GroupArgs<T> a, const T *__restrict__ X, T *__restrict__ Y) {
    if (a.skip && *a.skip) return;
    constexpr int RG = kGroupRows;
    __shared__ __align__(16) T cs[2][kGroupChunk][RG];
    __shared__ int js[2][kGroupChunk];
    __shared__ int sg[17];
    const int g = blockIdx.x, tid = threadIdx.x, len = a.len;
    const int r0 = g * RG, nr = min(RG, a.rows - r0);
    const int c0 = blockIdx.y * (NT * ITEMS);
    const int u0 = a.uoff[g], u1 = a.uoff[g + 1];
    if (tid < 17) sg[tid] = a.useg[(size_t)g * 17 + tid];
    auto stage = [&](int u, int b) {
        const int n = min(kGroupChunk, u1 - u);
        // coefficient rows are RG * sizeof(T) bytes: 16-byte pieces
        constexpr int per = RG * (int)sizeof(T) / 16;
        for (int idx = tid; idx < n * per; idx += NT)
            __pipeline_memcpy_async(reinterpret_cast<char *>(&cs[b][0][0]) + 16 * idx,
                                    reinterpret_cast<const char *>(a.coef + (size_t)u * RG) +
                                        16 * idx,
                                    16);
        for (int idx = tid; idx < n; idx += NT) js[b][idx] = a.uidx[u + idx];
        __pipeline_commit();
    };
    T acc[RG][ITEMS];
#pragma unroll
    for (int r = 0; r < RG; r++)
#pragma unroll
        for (int i = 0; i < ITEMS; i++) acc[r][i] = T(0);
    int col[ITEMS];
    bool in[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        col[i] = c0 + tid + NT * i;
        in[i] = col[i] < len;
    }
    if (u0 < u1) stage(u0, 0);
    int b = 0;
    for (int u = u0; u < u1; u += kGroupChunk, b ^= 1) {
        __pipeline_wait_prior(0);
        __syncthreads();  // chunk b landed; every thread is done with chunk b^1
        if (u + kGroupChunk < u1) stage(u + kGroupChunk, b ^ 1);
        const int ue = min(u + kGroupChunk, u1);
#define JCI_CLASS(QM)                                                                   \
    {                                                                                   \
        const int lo = max(sg[QM], u), hi = min(sg[QM + 1], ue);                        \
        if (lo < hi)                                                                    \
            group_class<T, ITEMS, QM>(acc, X, cs[b], js[b], col, in, len, lo - u, hi - u); \
    }
        JCI_CLASS(1)
        JCI_CLASS(2)
        JCI_CLASS(3)
        JCI_CLASS(4)
        JCI_CLASS(5)
        JCI_CLASS(6)
        JCI_CLASS(7)
        JCI_CLASS(8)
        JCI_CLASS(9)
        JCI_CLASS(10)
        JCI_CLASS(11)
        JCI_CLASS(12)
        JCI_CLASS(13)
        JCI_CLASS(14)
        JCI_CLASS(15)
#undef JCI_CLASS
    }
#pragma unroll
    for (int r = 0; r < RG; r++) {
        if (r < nr) {
            const long long o = (long long)(r0 + r) * len;
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                if (!in[i]) continue;
                T v = acc[r][i];
                if (a.hd) v = fma(a.hd[o + col[i]], X[o + col[i]], v);
                if (a.add) v += Y[o + col[i]];
                Y[o + col[i]] = v;
            }
        }
    }
}

// The same sums for small spaces, where one thread per column leaves the
// SMs nearly idle (FCI(12,12): 58 groups x 4 segments of 256 columns).
// Here the W warps of a CTA share its 32 ITEMS columns (lane + 32 i) and
// split the group's union: within every staged chunk, warp w takes the
// entry quads whose index in the chunk is w mod W.  The W partial sums of
// each output are then added in shared memory in warp order, so results
// stay bitwise reproducible.
constexpr int kSplitWarps = 4;

template <typename T, int ITEMS>
__device__ __forceinline__ void group_split(const GroupArgs<T> &a, const T *__restrict__ X,
                                            T *__restrict__ Y) {
    if (a.skip && *a.skip) return;
    constexpr int RG = kGroupRows, W = kSplitWarps, NT = 32 * W, CW = 32 * ITEMS;
    constexpr size_t kStage = 2 * kGroupChunk * RG * sizeof(T) + 2 * kGroupChunk * sizeof(int);
    constexpr size_t kRed = (size_t)W * RG * CW * sizeof(T);
    __shared__ __align__(16) unsigned char smem[kStage > kRed ? kStage : kRed];
    __shared__ int sg[17];
    T(*cs)[kGroupChunk][RG] = reinterpret_cast<T(*)[kGroupChunk][RG]>(smem);
    int(*js)[kGroupChunk] =
        reinterpret_cast<int(*)[kGroupChunk]>(smem + 2 * kGroupChunk * RG * sizeof(T));
    T *red = reinterpret_cast<T *>(smem);  // [W][RG][CW], after the last chunk
    const int g = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int len = a.len, r0 = g * RG, nr = min(RG, a.rows - r0);
    const int c0 = blockIdx.y * CW;
    const int u0 = a.uoff[g], u1 = a.uoff[g + 1];
    if (tid < 17) sg[tid] = a.useg[(size_t)g * 17 + tid];
    auto stage = [&](int u, int b) {
        const int n = min(kGroupChunk, u1 - u);
        constexpr int per = RG * (int)sizeof(T) / 16;
        for (int idx = tid; idx < n * per; idx += NT)
            __pipeline_memcpy_async(reinterpret_cast<char *>(&cs[b][0][0]) + 16 * idx,
                                    reinterpret_cast<const char *>(a.coef + (size_t)u * RG) +
                                        16 * idx,
                                    16);
        for (int idx = tid; idx < n; idx += NT) js[b][idx] = a.uidx[u + idx];
        __pipeline_commit();
    };
    T acc[RG][ITEMS];
#pragma unroll
    for (int r = 0; r < RG; r++)
#pragma unroll
        for (int i = 0; i < ITEMS; i++) acc[r][i] = T(0);
    int col[ITEMS];
    bool in[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        col[i] = c0 + lane + 32 * i;
        in[i] = col[i] < len;
    }
    if (u0 < u1) stage(u0, 0);
    int b = 0;
    for (int u = u0; u < u1; u += kGroupChunk, b ^= 1) {
        __pipeline_wait_prior(0);
        __syncthreads();  // chunk b landed; every thread is done with chunk b^1
        if (u + kGroupChunk < u1) stage(u + kGroupChunk, b ^ 1);
        const int ue = min(u + kGroupChunk, u1);
        // class QM's part of the chunk, [lo, hi) relative to u: this warp's
        // first quad is the first one at or after lo with index = warp mod W
#define JCI_CLASS(QM)                                                                  \
    {                                                                                  \
        const int lo = max(sg[QM], u) - u, hi = min(sg[QM + 1], ue) - u;               \
        if (lo < hi) {                                                                 \
            const int k0 = lo + 4 * ((warp - (lo >> 2) % W + W) % W);                   \
            if (k0 < hi)                                                               \
                group_class<T, ITEMS, QM, W>(acc, X, cs[b], js[b], col, in, len, k0, hi); \
        }                                                                              \
    }
        JCI_CLASS(1)
        JCI_CLASS(2)
        JCI_CLASS(3)
        JCI_CLASS(4)
        JCI_CLASS(5)
        JCI_CLASS(6)
        JCI_CLASS(7)
        JCI_CLASS(8)
        JCI_CLASS(9)
        JCI_CLASS(10)
        JCI_CLASS(11)
        JCI_CLASS(12)
        JCI_CLASS(13)
        JCI_CLASS(14)
        JCI_CLASS(15)
#undef JCI_CLASS
    }
    __syncthreads();  // the staging buffers become the reduction buffer
#pragma unroll
    for (int r = 0; r < RG; r++)
#pragma unroll
        for (int i = 0; i < ITEMS; i++) red[((size_t)warp * RG + r) * CW + lane + 32 * i] = acc[r][i];
    __syncthreads();
    for (int idx = tid; idx < RG * CW; idx += NT) {
        const int r = idx / CW, cc = idx - r * CW, c = c0 + cc;
        if (r >= nr || c >= len) continue;
        T v = red[idx];
#pragma unroll
        for (int w = 1; w < W; w++) v += red[(size_t)w * RG * CW + idx];
        const long long o = (long long)(r0 + r) * len + c;
        if (a.hd) v = fma(a.hd[o], X[o], v);
        if (a.add) v += Y[o];
        Y[o] = v;
    }
}

// Register bounds: the FP64 2-column form takes 136 registers unbounded (3
// CTAs per SM) and fits 128 without spills at 4 CTAs per SM.  The other
// forms keep the compiler's own choice: any bound there makes it spend
// registers on unrolling and lose occupancy (FP32 2-column: 66 unbounded,
// 96 or spills when bounded).
template <typename T, int ITEMS>
__global__ void __launch_bounds__(32 * kSplitWarps)
    k_sigma_group_split(GroupArgs<T> a, const T *__restrict__ X, T *__restrict__ Y) {
    group_split<T, ITEMS>(a, X, Y);
}
__global__ void __launch_bounds__(32 * kSplitWarps, 4)
    k_sigma_group_split_f64x2(GroupArgs<double> a, const double *__restrict__ X,
                              double *__restrict__ Y) {
    group_split<double, 2>(a, X, Y);
}

// coef[(uoff[g] + upos[f][s]) RG + s - g RG] = dblH[f][s] for every double f
// of every string s (g = s / RG); entries no double reaches stay zero.
template <typename T>
__global__ void k_group_coef(int nstr, int nd, const T *__restrict__ dblH,
                             const uint16_t *__restrict__ upos, const int *__restrict__ uoff,
                             T *__restrict__ coef) {
    const long long n = (long long)nstr * nd;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(e % nstr), g = s / kGroupRows;
        coef[((long long)uoff[g] + upos[e]) * kGroupRows + (s - g * kGroupRows)] = dblH[e];
    }
}

}  // namespace

// Host structure of the groups of one spin (integral-independent): the
// union of each group's double targets, sorted by class (the set of row
// quads that reach an entry, 1..15) and within a class by string, every
// class padded with zero-coefficient copies of its first entry to a
// multiple of 4; the class boundaries; every double's position in its
// group's union.  The coefficients are filled on the device (group_fill)
// from the current double values.
jci_status group_tables_build(const jci_space *s, int spin, GroupTables *t) {
    const SpinSpace &X = s->sp[spin];
    const int n = X.nstr, nd = X.max_doub, ng = (n + kGroupRows - 1) / kGroupRows;
    if (n < 1 || nd < 1) return JCI_ERR_SPACE;
    std::vector<int> uoff(ng + 1, 0), uidx, useg((size_t)ng * 17);
    std::vector<uint16_t> upos((size_t)nd * n);
    std::vector<int> u, list;
    for (int g = 0; g < ng; g++) {
        const int r0 = g * kGroupRows, r1 = std::min(n, r0 + kGroupRows);
        u.clear();
        for (int r = r0; r < r1; r++) {
            if (X.doff[r + 1] - X.doff[r] != nd) return JCI_ERR_SPACE;
            for (long long k = X.doff[r]; k < X.doff[r + 1]; k++) u.push_back(X.doub[k].target);
        }
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        // row quads reaching each entry
        std::vector<int> qm(u.size(), 0);
        for (int r = r0; r < r1; r++)
            for (int f = 0; f < nd; f++) {
                const int tgt = X.doub[X.doff[r] + f].target;
                qm[std::lower_bound(u.begin(), u.end(), tgt) - u.begin()] |= 1 << ((r - r0) / 4);
            }
        list.clear();
        std::vector<int> where(u.size());
        useg[(size_t)g * 17] = (int)uidx.size();
        for (int c = 1; c <= 15; c++) {
            useg[(size_t)g * 17 + c] = (int)(uidx.size() + list.size());
            const size_t first = list.size();
            for (size_t e = 0; e < u.size(); e++)
                if (qm[e] == c) {
                    where[e] = (int)(uidx.size() + list.size()) - uoff[g];
                    list.push_back(u[e]);
                }
            if (list.size() > first)
                while ((list.size() - first) % 4) list.push_back(list[first]);
        }
        useg[(size_t)g * 17 + 16] = (int)(uidx.size() + list.size());
        if (list.size() > 65535) return JCI_ERR_SPACE;
        for (int r = r0; r < r1; r++)
            for (int f = 0; f < nd; f++) {
                const int tgt = X.doub[X.doff[r] + f].target;
                upos[(size_t)f * n + r] =
                    (uint16_t)where[std::lower_bound(u.begin(), u.end(), tgt) - u.begin()];
            }
        uidx.insert(uidx.end(), list.begin(), list.end());
        uoff[g + 1] = (int)uidx.size();
    }
    GroupTables h;
    h.ng = ng;
    h.rows = n;
    h.nd = nd;
    h.nu = std::max<size_t>(uidx.size(), 1);
    uidx.resize(h.nu, 0);
    jci_status r = JCI_OK;
    if (cudaMalloc(&h.uoff, uoff.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h.uidx, uidx.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h.useg, useg.size() * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h.upos, upos.size() * sizeof(uint16_t)) != cudaSuccess ||
        cudaMalloc(&h.c64, h.nu * kGroupRows * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h.c32, h.nu * kGroupRows * sizeof(float)) != cudaSuccess)
        r = JCI_ERR_CUDA;
    if (!r && (cudaMemcpy(h.uoff, uoff.data(), uoff.size() * sizeof(int),
                          cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(h.uidx, uidx.data(), uidx.size() * sizeof(int),
                          cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(h.useg, useg.data(), useg.size() * sizeof(int),
                          cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(h.upos, upos.data(), upos.size() * sizeof(uint16_t),
                          cudaMemcpyHostToDevice) != cudaSuccess))
        r = JCI_ERR_CUDA;
    if (r) {
        group_tables_free(&h);
        return r;
    }
    *t = h;
    return JCI_OK;
}

void group_tables_free(GroupTables *t) {
    cudaFree(t->uoff);
    cudaFree(t->uidx);
    cudaFree(t->useg);
    cudaFree(t->upos);
    cudaFree(t->c64);
    cudaFree(t->c32);
    *t = GroupTables();
}

// Coefficient blocks from the current double values ([double][string], FP64
// and FP32), on stream st.
jci_status group_fill(GroupTables *t, const double *dblH, const float *dblHf, cudaStream_t st) {
    JCI_CUDA(cudaMemsetAsync(t->c64, 0, t->nu * kGroupRows * sizeof(double), st));
    JCI_CUDA(cudaMemsetAsync(t->c32, 0, t->nu * kGroupRows * sizeof(float), st));
    const long long n = (long long)t->rows * t->nd;
    const int grid = (int)std::min<long long>((n + 255) / 256, 4096);
    k_group_coef<double><<<grid, 256, 0, st>>>(t->rows, t->nd, dblH, t->upos, t->uoff, t->c64);
    k_group_coef<float><<<grid, 256, 0, st>>>(t->rows, t->nd, dblHf, t->upos, t->uoff, t->c32);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

// Variants 1 and 2: one thread per column with `variant` columns each, in
// 256-thread CTAs, or 128-thread ones when the wider CTAs would give fewer
// than four per SM.  Variants 3 and 4: the union split over the warps of a
// CTA (k_sigma_group_split) with 2 and 1 columns per lane.
template <typename T>
jci_status group_launch(const GroupArgs<T> &a, int variant, int device, const T *x, T *y,
                        cudaStream_t st) {
    if (variant < 1 || variant > 4) return JCI_ERR_ARG;
    if (variant >= 3) {
        const int ng = (a.rows + kGroupRows - 1) / kGroupRows, cw = variant == 3 ? 64 : 32;
        const dim3 grid(ng, (a.len + cw - 1) / cw);
        if constexpr (sizeof(T) == sizeof(double)) {
            if (variant == 3)
                k_sigma_group_split_f64x2<<<grid, 32 * kSplitWarps, 0, st>>>(a, x, y);
        } else {
            if (variant == 3)
                k_sigma_group_split<T, 2><<<grid, 32 * kSplitWarps, 0, st>>>(a, x, y);
        }
        if (variant == 4)
            k_sigma_group_split<T, 1><<<grid, 32 * kSplitWarps, 0, st>>>(a, x, y);
        JCI_CUDA(cudaGetLastError());
        return JCI_OK;
    }
    const int items = variant;
    int nsm = 0;
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    const int ng = (a.rows + kGroupRows - 1) / kGroupRows;
    const long long wide = (long long)ng * ((a.len + 256 * items - 1) / (256 * items));
    const int nt = wide < 4LL * nsm ? 128 : 256;
    const int seg = nt * items;
    const dim3 grid(ng, (a.len + seg - 1) / seg);
#define JCI_GROUP(NT, IT) \
    if (nt == NT && items == IT) k_sigma_group<T, NT, IT><<<grid, NT, 0, st>>>(a, x, y);
    JCI_GROUP(128, 1)
    JCI_GROUP(128, 2)
    JCI_GROUP(256, 1)
    JCI_GROUP(256, 2)
#undef JCI_GROUP
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

template jci_status group_launch<double>(const GroupArgs<double> &, int, int, const double *,
                                         double *, cudaStream_t);
template jci_status group_launch<float>(const GroupArgs<float> &, int, int, const float *, float *,
                                        cudaStream_t);

}  // namespace jci
