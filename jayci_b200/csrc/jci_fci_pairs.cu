// jci_fci_pairs.cu -- same-spin doubles of the one-group sigma through
// (N-2)-electron hole strings (hmatels_2xaa / hmatels_2xbb,
// mpi_source/action_util.c:237-245).
//
// In a one-group space every same-spin double I <- J (the strings differ in
// two orbitals) has exactly one hole string K = I n J with N - 2 electrons.
// With I = K + {i,j}, J = K + {k,l} (i < j, k < l, {i,j} n {k,l} empty),
//   <I|H|J> = phi(K;i,j) phi(K;k,l) [(ik|jl) - (il|jk)],
// phi(K;k,l) = (-1)^(#K below k + #K below l), the phase of a+_k a+_l |K>.
// So the strings K + p over the pairs p of K's free orbitals form a dense
// block, and with W[P][Q] = (ik|jl) - (il|jk) over orbital pairs (zero when
// the pairs overlap) and W_K[p][q] = phi_p phi_q W[p][q]:
//   E[K][p][c] = sum_q W_K[p][q] X[K + q][c]        (phase 1, dense products)
//   Y[I][c]    = sum_{K in I} E[K][I - K][c]          (phase 2, C(N,2) rows)
// At FCI(16,16): 8008 hole strings with 45 pairs each (1260 of the 2025
// block entries are doubles), against the string-group form's 16 x 3.7
// reached rows per union entry.  Phase 1 runs in FP64 on the FP64 tensor
// cores (mma.sync m8n8k4) and in FP32 on the FMA pipes; E is kept for one
// block of columns at a time.  Every sum runs in a fixed order: bitwise
// reproducible.
#include <cuda_pipeline.h>

#include <algorithm>
#include <unordered_map>
#include <vector>

#include "jci_internal.h"
#include "jci_kernels.cuh"

namespace jci {

namespace {

constexpr int kPairThreads = 256;
constexpr int kPairCols = 64;      // columns per staged chunk
constexpr int kPullRows = 8;       // strings per CTA of the pull
constexpr size_t kPairEBytes = size_t(1) << 30;  // E of the widest column block
constexpr size_t kPairEBytesWide = size_t(4) << 30;  // the same for variant 7

template <typename T>
struct PairArgs {
    int nk, np, NP, ngp, nt;   // hole strings, pairs (padded), orbital pairs, holes per string
    int rows, len;             // strings of this spin x row length
    const int *jrow;           // [K][p] source string | phase << 31
    const uint16_t *gp;        // [K][p] orbital pair
    const int *pull;           // [I][t] K * np + p
    const T *W;                // [ngp][ngp]
    const int *skip;
};

__device__ __forceinline__ void pair_dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// Shared-memory strides: rows of W_K and of the staged chunk padded so that
// the FP64 fragment loads (4 rows x 8 consecutive elements) hit distinct banks.
template <typename T>
__host__ __device__ constexpr int pair_ws(int NP) { return NP + (sizeof(T) == 8 ? 4 : 1); }
template <typename T>
__host__ __device__ constexpr int pair_ds() { return kPairCols + (sizeof(T) == 8 ? 4 : 0); }

template <typename T>
size_t pair_smem(int NP) {
    return ((size_t)NP * pair_ws<T>(NP) + 2 * (size_t)NP * pair_ds<T>()) * sizeof(T) +
           (size_t)NP * sizeof(int) + 16;
}

// Phase 1 for hole string blockIdx.x and the columns [c0, c0 + cb) of the
// row length: E[(K np + p) cb + c - c0].  NP = 16 RT padded pairs.
template <typename T, int RT>
__global__ void __launch_bounds__(kPairThreads)
    k_pairs_product(PairArgs<T> a, const T *__restrict__ X, T *__restrict__ E, int c0, int cb) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NP = 16 * RT;
    constexpr int WS = pair_ws<T>(NP), DS = pair_ds<T>();
    T *Ws = reinterpret_cast<T *>(smem_raw);            // [NP][WS]
    T *Ds = Ws + (size_t)NP * WS;                       // [2][NP][DS]
    int *jr = reinterpret_cast<int *>(Ds + 2 * (size_t)NP * DS);  // [NP]
    const int tid = threadIdx.x, K = blockIdx.x, np = a.np;
    const long long kb = (long long)K * np;
    for (int p = tid; p < NP; p += kPairThreads) jr[p] = p < np ? a.jrow[kb + p] : 0;
    __syncthreads();
    for (int idx = tid; idx < NP * NP; idx += kPairThreads) {
        const int p = idx / NP, q = idx - p * NP;
        T v = T(0);
        if (p < np && q < np) {
            v = a.W[(size_t)a.gp[kb + p] * a.ngp + a.gp[kb + q]];
            if ((jr[p] ^ jr[q]) < 0) v = -v;  // phi_p phi_q
        }
        Ws[p * WS + q] = v;
    }
    const int c1 = min(a.len, c0 + cb);
    auto stage = [&](int c, T *buf) {
        for (int idx = tid; idx < NP * kPairCols; idx += kPairThreads) {
            const int q = idx >> 6, cc = idx & 63;
            T *dst = buf + q * DS + cc;
            if (q < np && c + cc < c1)
                __pipeline_memcpy_async(dst, X + (long long)(jr[q] & 0x7fffffff) * a.len + c + cc,
                                        sizeof(T));
            else
                *dst = T(0);
        }
        __pipeline_commit();
    };
    const size_t dsz = (size_t)NP * DS;
    const int nchunk = (c1 - c0 + kPairCols - 1) / kPairCols;
    stage(c0, Ds);
    for (int ci = 0; ci < nchunk; ci++) {
        const int c = c0 + ci * kPairCols;
        const T *Dc = Ds + (ci & 1) * dsz;
        if (ci + 1 < nchunk) {
            stage(c + kPairCols, Ds + ((ci + 1) & 1) * dsz);
            __pipeline_wait_prior(1);
        } else {
            __pipeline_wait_prior(0);
        }
        __syncthreads();
        if constexpr (sizeof(T) == 8) {
            // warp w: columns 16 (w & 3) .. + 15, pair rows 8 RT (w >> 2) .. + 8 RT - 1
            const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
            const int wn = warp & 3, wm = warp >> 2;
            double acc[RT][2][2];
#pragma unroll
            for (int i = 0; i < RT; i++)
#pragma unroll
                for (int n = 0; n < 2; n++) acc[i][n][0] = acc[i][n][1] = 0.0;
            const double *ap = Ws + (size_t)(8 * RT * wm + g) * WS + t;
            const double *bp = Dc + t * DS + 16 * wn + g;
#pragma unroll 4
            for (int k0 = 0; k0 < NP; k0 += 4) {
                const double b0 = bp[k0 * DS], b1 = bp[k0 * DS + 8];
#pragma unroll
                for (int i = 0; i < RT; i++) {
                    const double av = ap[8 * i * WS + k0];
                    pair_dmma(acc[i][0], av, b0);
                    pair_dmma(acc[i][1], av, b1);
                }
            }
            // lane holds row g, columns 2t and 2t+1 of each 8 x 8 tile
#pragma unroll
            for (int i = 0; i < RT; i++) {
                const int p = 8 * (RT * wm + i) + g;
                if (p >= np) continue;
#pragma unroll
                for (int n = 0; n < 2; n++) {
                    const int cc = c - c0 + 16 * wn + 8 * n + 2 * t;
                    double *dst = E + (size_t)(kb + p) * cb + cc;
                    if (c0 + cc + 1 < c1)
                        *reinterpret_cast<double2 *>(dst) = make_double2(acc[i][n][0], acc[i][n][1]);
                    else if (c0 + cc < c1)
                        dst[0] = acc[i][n][0];
                }
            }
        } else {
            // 16 x 16 threads: rows ty RT .. + RT - 1, columns tx + 16 j
            const int tx = tid & 15, ty = tid >> 4;
            T acc[RT][4];
#pragma unroll
            for (int i = 0; i < RT; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = T(0);
#pragma unroll 4
            for (int k = 0; k < NP; k++) {
                const T *br = Dc + k * DS + tx;
                const T b0 = br[0], b1 = br[16], b2 = br[32], b3 = br[48];
#pragma unroll
                for (int i = 0; i < RT; i++) {
                    const T av = Ws[(ty * RT + i) * WS + k];
                    acc[i][0] = fma(av, b0, acc[i][0]);
                    acc[i][1] = fma(av, b1, acc[i][1]);
                    acc[i][2] = fma(av, b2, acc[i][2]);
                    acc[i][3] = fma(av, b3, acc[i][3]);
                }
            }
#pragma unroll
            for (int i = 0; i < RT; i++) {
                const int p = ty * RT + i;
                if (p >= np) continue;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int cc = c - c0 + tx + 16 * j;
                    if (c0 + cc < c1) E[(size_t)(kb + p) * cb + cc] = acc[i][j];
                }
            }
        }
        __syncthreads();
    }
}

// Phase 2: Y[I][c] = sum_t E[pull[I][t]][c - c0] (+ hd X, + Y) for the
// strings I of CTA row block blockIdx.x and the columns c0 + 256 blockIdx.y + tid.
template <typename T>
__global__ void __launch_bounds__(kPairThreads)
    k_pairs_pull(PairArgs<T> a, const T *__restrict__ E, const T *__restrict__ X,
                 T *__restrict__ Y, const T *__restrict__ hd, int add, int c0, int cb) {
    if (a.skip && *a.skip) return;
    extern __shared__ int pl[];  // [kPullRows][nt]
    const int r0 = blockIdx.x * kPullRows, nr = min(kPullRows, a.rows - r0), nt = a.nt;
    for (int idx = threadIdx.x; idx < nr * nt; idx += kPairThreads)
        pl[idx] = a.pull[(size_t)r0 * nt + idx];
    __syncthreads();
    const int cc = blockIdx.y * kPairThreads + threadIdx.x, c = c0 + cc;
    if (cc >= cb || c >= a.len) return;
    for (int r = 0; r < nr; r++) {
        const int *pr = pl + r * nt;
        T v = T(0);
        int t = 0;
        for (; t + 4 <= nt; t += 4) {  // four loads in flight, added in order
            const T e0 = E[(size_t)pr[t] * cb + cc], e1 = E[(size_t)pr[t + 1] * cb + cc];
            const T e2 = E[(size_t)pr[t + 2] * cb + cc], e3 = E[(size_t)pr[t + 3] * cb + cc];
            v += e0;
            v += e1;
            v += e2;
            v += e3;
        }
        for (; t < nt; t++) v += E[(size_t)pr[t] * cb + cc];
        const long long o = (long long)(r0 + r) * a.len + c;
        if (hd) v = fma(hd[o], X[o], v);
        if (add) v += Y[o];
        Y[o] = v;
    }
}

template <typename T>
using PairKernel = void (*)(PairArgs<T>, const T *, T *, int, int);

template <typename T>
PairKernel<T> pair_kernel(int RT) {
    switch (RT) {
        case 1: return k_pairs_product<T, 1>;
        case 2: return k_pairs_product<T, 2>;
        case 3: return k_pairs_product<T, 3>;
        case 4: return k_pairs_product<T, 4>;
        case 5: return k_pairs_product<T, 5>;
        default: return nullptr;
    }
}

// ---- singles through (N-1)-electron hole strings ---------------------------
//
// Every single I <- J of a one-group space (one electron moved) has exactly
// one hole string K = I n J with N - 1 electrons; with I = K + k, J = K + l
// the element is s (a1(K;k,l) + jc[(kl)][c]), the one-body part a1 depending
// only on K and (k,l) and jc on the column's string of the other spin.  So
//   E[K][k][c] = sum_{l != k} s_kl (a1_kl + jc[(kl)][c]) X[K + l][c]
//   Y[I][c]    = sum_{K in I} E[K][I - K][c]            (N rows per string)
// which reads each source row once per hole string (N - 1 + 1 free orbitals
// share it) instead of once per single.  Phase 2 is k_pairs_pull.
constexpr int kHsMaxFree = 16;   // free orbitals of a hole string
constexpr int kHsPerCta = 32;    // hole strings per CTA of phase 1

template <typename T>
struct HsArgs {
    int nk, nf, len, npair;
    const int *srow;        // [K][x] string K + free orbital x
    const T *a1s;           // [K][x][y] s (a1 of the single K+x <- K+y), 0 on the diagonal
    const uint16_t *pp;     // [K][x][y] pair index of the single | phase << 15
    const T *jc;            // [pair][column] Coulomb part
    const int *skip;
};

// Phase 1 for hole strings blockIdx.x * kHsPerCta.. and the 64 columns
// c0 + 64 blockIdx.y.. of the block [c0, c0 + cb): the jc chunk of every
// pair is staged in shared memory once per CTA; thread (column, lane)
// takes every fourth hole string of the CTA.
template <typename T>
__global__ void __launch_bounds__(256)
    k_hsingles_product(HsArgs<T> a, const T *__restrict__ X, T *__restrict__ E, int c0, int cb) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *Js = reinterpret_cast<T *>(smem_raw);  // [npair][64]
    const int tid = threadIdx.x, col = tid & 63, lane = tid >> 6;
    const int cc = blockIdx.y * kPairCols + col, c = c0 + cc;
    const int c1 = min(a.len, c0 + cb);
    const bool ok = c < c1;
    for (int idx = tid; idx < a.npair * kPairCols; idx += 256) {
        const int q = idx >> 6, k = idx & 63, cq = c0 + blockIdx.y * kPairCols + k;
        Js[idx] = cq < c1 ? a.jc[(long long)q * a.len + cq] : T(0);
    }
    __syncthreads();
    const int nf = a.nf;
    for (int kk = lane; kk < kHsPerCta; kk += 4) {
        const int K = blockIdx.x * kHsPerCta + kk;
        if (K >= a.nk) break;
        T xv[kHsMaxFree];
#pragma unroll
        for (int x = 0; x < kHsMaxFree; x++)
            xv[x] = (x < nf && ok) ? X[(long long)a.srow[(size_t)K * nf + x] * a.len + c] : T(0);
        const size_t qb = (size_t)K * nf * nf;
        for (int x = 0; x < nf; x++) {
            T acc = T(0);
#pragma unroll
            for (int y = 0; y < kHsMaxFree; y++) {
                if (y >= nf || y == x) continue;
                const size_t q = qb + x * nf + y;
                const uint16_t pq = a.pp[q];
                const T j = Js[(pq & 0x7fff) * kPairCols + col];
                acc += (a.a1s[q] + ((pq >> 15) ? -j : j)) * xv[y];
            }
            if (ok) E[((size_t)K * nf + x) * cb + cc] = acc;
        }
    }
}

// a1s from the current one-body parts: a1s[q] = s a1T[single][string].
template <typename T>
__global__ void k_hs_fill(long long n, const int *__restrict__ sidx, const T *__restrict__ a1T,
                          T *__restrict__ a1s) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int e = sidx[q];
        T v = T(0);
        if (e != -1) {
            v = a1T[e & 0x7fffffff];
            if (e < 0) v = -v;
        }
        a1s[q] = v;
    }
}

}  // namespace

// Tables of one spin: the hole strings K (the (N-2)-subsets of the varying
// orbitals, lexical), per K its free pairs in lexical order with their
// source strings, phases and orbital pairs, and per string its C(N,2) hole
// strings in the lexical order of the removed pairs.  JCI_ERR_SPACE when the
// spin's strings are not every N-subset of one orbital set plus orbitals
// common to all of them, or when there are no doubles.
jci_status pair_tables_build(const jci_space *s, int spin, PairTables *t) {
    const SpinSpace &X = s->sp[spin];
    const int ns = X.nstr, ne = X.nelec;
    if (ns < 1 || ne < 2) return JCI_ERR_SPACE;
    uint64_t uni = 0, all = ~0ull;
    for (int i = 0; i < ns; i++) {
        uint64_t m = 0;
        for (int e = 0; e < ne; e++) {
            const int o = X.istr[(size_t)i * ne + e];
            if (o < 1 || o > 64) return JCI_ERR_SPACE;
            m |= 1ull << (o - 1);
        }
        uni |= m;
        all &= m;
    }
    std::vector<int> orb, fixed;  // varying orbitals, orbitals of every string (1-based)
    for (int o = 1; o <= 64; o++) {
        if ((all >> (o - 1)) & 1) fixed.push_back(o);
        else if ((uni >> (o - 1)) & 1) orb.push_back(o);
    }
    const int no = (int)orb.size(), nv = ne - (int)fixed.size();
    if (nv < 2 || no - nv < 2 || binom(no, nv) != ns) return JCI_ERR_SPACE;
    const int nf = no - nv + 2;  // free orbitals of a hole string
    const int np = nf * (nf - 1) / 2, NP = (np + 15) / 16 * 16;
    if (NP > 80) return JCI_ERR_SPACE;
    const long long nk = binom(no, nv - 2);
    const int nt = nv * (nv - 1) / 2, ngp = no * (no - 1) / 2;
    if (nk * np >= (1ll << 31)) return JCI_ERR_SPACE;
    // hole strings as masks over the positions of orb, in lexical order
    std::vector<uint64_t> kmask;
    std::unordered_map<uint64_t, int> krank;
    {
        std::vector<int> c(nv - 2);
        for (int i = 0; i < nv - 2; i++) c[i] = i;
        for (;;) {
            uint64_t m = 0;
            for (int x : c) m |= 1ull << x;
            krank[m] = (int)kmask.size();
            kmask.push_back(m);
            int i = nv - 3;
            while (i >= 0 && c[i] == no - (nv - 2) + i) i--;
            if (i < 0) break;
            c[i]++;
            for (int j = i + 1; j < nv - 2; j++) c[j] = c[j - 1] + 1;
        }
    }
    auto gpair = [&](int a, int b) { return a * (2 * no - a - 1) / 2 + (b - a - 1); };
    std::vector<int> jrow((size_t)nk * np), pull((size_t)ns * nt);
    std::vector<uint16_t> gp((size_t)nk * np);
    std::vector<int> o(ne), F;
    for (long long k = 0; k < nk; k++) {
        const uint64_t m = kmask[k];
        F.clear();
        for (int x = 0; x < no; x++)
            if (!((m >> x) & 1)) F.push_back(x);
        int p = 0;
        for (int u = 0; u < nf; u++)
            for (int v = u + 1; v < nf; v++, p++) {
                const int ka = F[u], la = F[v];
                // string K + {ka, la} (with the fixed orbitals) and its phase
                int n = 0, below = 0;
                for (int f : fixed) {
                    o[n++] = f;
                    below += (f < orb[ka]) + (f < orb[la]);
                }
                for (int x = 0; x < no; x++)
                    if (((m >> x) & 1) || x == ka || x == la) o[n++] = orb[x];
                for (int x = 0; x < no; x++)
                    if ((m >> x) & 1) below += (x < ka) + (x < la);
                std::sort(o.begin(), o.end());
                const int J = string_index(s, spin, o.data());
                if (J < 0) return JCI_ERR_SPACE;
                jrow[(size_t)k * np + p] = J | ((below & 1) ? (int)0x80000000u : 0);
                gp[(size_t)k * np + p] = (uint16_t)gpair(ka, la);
            }
    }
    std::vector<int> orbpos(65, -1);
    for (int x = 0; x < no; x++) orbpos[orb[x]] = x;
    for (int i = 0; i < ns; i++) {
        uint64_t m = 0;
        std::vector<int> vp;
        for (int e = 0; e < ne; e++) {
            const int x = orbpos[X.istr[(size_t)i * ne + e]];
            if (x >= 0) {
                m |= 1ull << x;
                vp.push_back(x);
            }
        }
        int t2 = 0;
        for (int u = 0; u < nv; u++)
            for (int v = u + 1; v < nv; v++, t2++) {
                const uint64_t km = m & ~(1ull << vp[u]) & ~(1ull << vp[v]);
                const auto it = krank.find(km);
                if (it == krank.end()) return JCI_ERR_SPACE;
                // rank of the pair (vp[u], vp[v]) among the free pairs of K
                int fu = 0, fv = 0;
                for (int x = 0; x < vp[u]; x++) fu += !((km >> x) & 1);
                for (int x = 0; x < vp[v]; x++) fv += !((km >> x) & 1);
                const int p = fu * (2 * nf - fu - 1) / 2 + (fv - fu - 1);
                pull[(size_t)i * nt + t2] = it->second * np + p;
            }
    }
    t->nk = (int)nk; t->np = np; t->NP = NP; t->nt = nt; t->ngp = ngp; t->rows = ns;
    t->orb = orb;
    JCI_CUDA(cudaMalloc(&t->jrow, jrow.size() * sizeof(int)));
    JCI_CUDA(cudaMalloc(&t->gp, gp.size() * sizeof(uint16_t)));
    JCI_CUDA(cudaMalloc(&t->pull, pull.size() * sizeof(int)));
    JCI_CUDA(cudaMalloc(&t->W64, (size_t)ngp * ngp * sizeof(double)));
    JCI_CUDA(cudaMalloc(&t->W32, (size_t)ngp * ngp * sizeof(float)));
    JCI_CUDA(cudaMemcpy(t->jrow, jrow.data(), jrow.size() * sizeof(int), cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(t->gp, gp.data(), gp.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(t->pull, pull.data(), pull.size() * sizeof(int), cudaMemcpyHostToDevice));
    return JCI_OK;
}

// W over the orbital pairs from the current integrals (the host copy that
// the device integrals are made from): W[(ij)][(kl)] = (ik|jl) - (il|jk),
// zero when the pairs share an orbital.
jci_status pair_fill(const jci_space *s, PairTables *t, cudaStream_t st) {
    const int no = (int)t->orb.size(), ngp = t->ngp;
    std::vector<int> pa(ngp), pb(ngp);
    for (int a = 0, P = 0; a < no; a++)
        for (int b = a + 1; b < no; b++, P++) {
            pa[P] = t->orb[a];
            pb[P] = t->orb[b];
        }
    t->w64.assign((size_t)ngp * ngp, 0.0);
    t->w32.assign((size_t)ngp * ngp, 0.f);
    const double *m2 = s->m2.data();
    for (int P = 0; P < ngp; P++)
        for (int Q = 0; Q < ngp; Q++) {
            const int i = pa[P], j = pb[P], k = pa[Q], l = pb[Q];
            if (i == k || i == l || j == k || j == l) continue;
            const double w = m2[eri_index(pair_index(i, k), pair_index(j, l))] -
                             m2[eri_index(pair_index(i, l), pair_index(j, k))];
            t->w64[(size_t)P * ngp + Q] = w;
            t->w32[(size_t)P * ngp + Q] = (float)w;
        }
    JCI_CUDA(cudaMemcpyAsync(t->W64, t->w64.data(), t->w64.size() * sizeof(double),
                             cudaMemcpyHostToDevice, st));
    JCI_CUDA(cudaMemcpyAsync(t->W32, t->w32.data(), t->w32.size() * sizeof(float),
                             cudaMemcpyHostToDevice, st));
    return JCI_OK;
}

void pair_tables_free(PairTables *t) {
    cudaFree(t->jrow);
    cudaFree(t->gp);
    cudaFree(t->pull);
    cudaFree(t->W64);
    cudaFree(t->W32);
    *t = PairTables();
}

size_t pair_smem_bytes(const PairTables &t, int prec) {
    return prec == 0 ? pair_smem<double>(t.NP) : pair_smem<float>(t.NP);
}

// Columns per block of phase 1 / phase 2: variant 5 the widest block whose E
// fits kPairEBytes (variant 7: kPairEBytesWide, fewer launches and W_K
// builds for more memory), variant 6 one 64-column chunk (E small enough
// for L2 at the mid sizes).
int pair_block_cols(const PairTables &t, int len, int variant, size_t w) {
    const int full = (len + kPairCols - 1) / kPairCols * kPairCols;
    if (variant == 6) return kPairCols;
    const size_t per_col = (size_t)t.nk * t.np * w;
    const int cb = (int)std::min<size_t>(full, (variant == 7 ? kPairEBytesWide : kPairEBytes) / per_col / kPairCols * kPairCols);
    return std::max(cb, kPairCols);
}

template <typename T>
jci_status pair_launch(const PairTables &t, int len, int variant, const T *x, T *y, const T *hd,
                       int add, const int *skip, T *E, int device, cudaStream_t st) {
    PairArgs<T> a;
    a.nk = t.nk; a.np = t.np; a.NP = t.NP; a.ngp = t.ngp; a.nt = t.nt;
    a.rows = t.rows; a.len = len;
    a.jrow = t.jrow; a.gp = t.gp; a.pull = t.pull;
    if constexpr (sizeof(T) == 8) a.W = t.W64;
    else a.W = t.W32;
    a.skip = skip;
    PairKernel<T> kern = pair_kernel<T>(t.NP / 16);
    if (!kern) return JCI_ERR_SPACE;
    const size_t smem = pair_smem<T>(t.NP);
    int optin = 0;
    JCI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    if (smem > (size_t)optin) return JCI_ERR_SPACE;
    JCI_CUDA(smem_optin(kern));
    const int cb = pair_block_cols(t, len, variant, sizeof(T));
    const size_t psmem = (size_t)kPullRows * t.nt * sizeof(int);
    for (int c0 = 0; c0 < len; c0 += cb) {
        kern<<<t.nk, kPairThreads, smem, st>>>(a, x, E, c0, cb);
        const int w = std::min(cb, len - c0);
        dim3 g((t.rows + kPullRows - 1) / kPullRows, (w + kPairThreads - 1) / kPairThreads);
        k_pairs_pull<T><<<g, kPairThreads, psmem, st>>>(a, E, x, y, hd, add, c0, cb);
    }
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

template jci_status pair_launch<double>(const PairTables &, int, int, const double *, double *,
                                        const double *, int, const int *, double *, int,
                                        cudaStream_t);
template jci_status pair_launch<float>(const PairTables &, int, int, const float *, float *,
                                       const float *, int, const int *, float *, int,
                                       cudaStream_t);

// Single tables of one spin through its (N-1)-electron hole strings, in the
// layout of the pair tables: hole strings in lexical order of the varying
// orbitals, free orbitals ascending, per string its N - f hole strings in
// ascending order of the removed orbital.  The coefficient of each ordered
// free pair (x, y) is the string K + x's single with target K + y (its
// position in the [single][string] one-body table, its phase, its pair).
jci_status hs_tables_build(const jci_space *s, int spin, HsTables *t) {
    const SpinSpace &X = s->sp[spin];
    const int ns = X.nstr, ne = X.nelec;
    if (ns < 1 || ne < 1) return JCI_ERR_SPACE;
    uint64_t uni = 0, all = ~0ull;
    for (int i = 0; i < ns; i++) {
        uint64_t m = 0;
        for (int e = 0; e < ne; e++) {
            const int o = X.istr[(size_t)i * ne + e];
            if (o < 1 || o > 64) return JCI_ERR_SPACE;
            m |= 1ull << (o - 1);
        }
        uni |= m;
        all &= m;
    }
    std::vector<int> orb, fixed;
    for (int o = 1; o <= 64; o++) {
        if ((all >> (o - 1)) & 1) fixed.push_back(o);
        else if ((uni >> (o - 1)) & 1) orb.push_back(o);
    }
    const int no = (int)orb.size(), nv = ne - (int)fixed.size();
    if (nv < 1 || no - nv < 1 || binom(no, nv) != ns) return JCI_ERR_SPACE;
    const int nf = no - nv + 1;
    if (nf > 16) return JCI_ERR_SPACE;
    const long long nk = binom(no, nv - 1);
    if (nk * nf * nf >= (1ll << 31)) return JCI_ERR_SPACE;
    for (int i = 0; i < ns; i++)
        if (X.soff[i + 1] - X.soff[i] != (long long)nv * (no - nv)) return JCI_ERR_SPACE;
    std::vector<uint64_t> kmask;
    std::unordered_map<uint64_t, int> krank;
    {
        std::vector<int> c(nv - 1);
        for (int i = 0; i < nv - 1; i++) c[i] = i;
        for (;;) {
            uint64_t m = 0;
            for (int x : c) m |= 1ull << x;
            krank[m] = (int)kmask.size();
            kmask.push_back(m);
            int i = nv - 2;
            while (i >= 0 && c[i] == no - (nv - 1) + i) i--;
            if (i < 0) break;
            c[i]++;
            for (int j = i + 1; j < nv - 1; j++) c[j] = c[j - 1] + 1;
        }
    }
    std::vector<int> srow((size_t)nk * nf), sidx((size_t)nk * nf * nf, -1), pull((size_t)ns * nv);
    std::vector<uint16_t> pp((size_t)nk * nf * nf, 0);
    std::vector<int> o(ne), F;
    for (long long k = 0; k < nk; k++) {
        const uint64_t m = kmask[k];
        F.clear();
        for (int x = 0; x < no; x++)
            if (!((m >> x) & 1)) F.push_back(x);
        for (int x = 0; x < nf; x++) {
            int n = 0;
            for (int f : fixed) o[n++] = f;
            for (int y = 0; y < no; y++)
                if (((m >> y) & 1) || y == F[x]) o[n++] = orb[y];
            std::sort(o.begin(), o.end());
            const int I = string_index(s, spin, o.data());
            if (I < 0) return JCI_ERR_SPACE;
            srow[(size_t)k * nf + x] = I;
        }
        for (int x = 0; x < nf; x++) {
            const int I = srow[(size_t)k * nf + x];
            for (int y = 0; y < nf; y++) {
                if (y == x) continue;
                const int J = srow[(size_t)k * nf + y];
                long long f = X.soff[I];
                while (f < X.soff[I + 1] && X.sing[f].target != J) f++;
                if (f == X.soff[I + 1]) return JCI_ERR_SPACE;
                const Exc &e = X.sing[f];
                const long long pos = (f - X.soff[I]) * ns + I;
                if (pos >= (1ll << 31) - 1) return JCI_ERR_SPACE;
                const size_t q = ((size_t)k * nf + x) * nf + y;
                sidx[q] = (int)pos | (e.sign < 0 ? (int)0x80000000u : 0);
                const int pr = pair_index(e.io0, e.fo0);
                if (pr >= 0x8000) return JCI_ERR_SPACE;
                pp[q] = (uint16_t)(pr | (e.sign < 0 ? 0x8000 : 0));
            }
        }
    }
    std::vector<int> orbpos(65, -1);
    for (int x = 0; x < no; x++) orbpos[orb[x]] = x;
    for (int i = 0; i < ns; i++) {
        uint64_t m = 0;
        std::vector<int> vp;
        for (int e = 0; e < ne; e++) {
            const int x = orbpos[X.istr[(size_t)i * ne + e]];
            if (x >= 0) {
                m |= 1ull << x;
                vp.push_back(x);
            }
        }
        for (int u = 0; u < nv; u++) {
            const uint64_t km = m & ~(1ull << vp[u]);
            const auto it = krank.find(km);
            if (it == krank.end()) return JCI_ERR_SPACE;
            int fx = 0;
            for (int x = 0; x < vp[u]; x++) fx += !((km >> x) & 1);
            pull[(size_t)i * nv + u] = it->second * nf + fx;
        }
    }
    t->nk = (int)nk; t->nf = nf; t->nt = nv; t->rows = ns;
    JCI_CUDA(cudaMalloc(&t->srow, srow.size() * sizeof(int)));
    JCI_CUDA(cudaMalloc(&t->sidx, sidx.size() * sizeof(int)));
    JCI_CUDA(cudaMalloc(&t->pp, pp.size() * sizeof(uint16_t)));
    JCI_CUDA(cudaMalloc(&t->pull, pull.size() * sizeof(int)));
    JCI_CUDA(cudaMalloc(&t->a1s64, sidx.size() * sizeof(double)));
    JCI_CUDA(cudaMalloc(&t->a1s32, sidx.size() * sizeof(float)));
    JCI_CUDA(cudaMemcpy(t->srow, srow.data(), srow.size() * sizeof(int), cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(t->sidx, sidx.data(), sidx.size() * sizeof(int), cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(t->pp, pp.data(), pp.size() * sizeof(uint16_t), cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(t->pull, pull.data(), pull.size() * sizeof(int), cudaMemcpyHostToDevice));
    return JCI_OK;
}

jci_status hs_fill(HsTables *t, const double *a1T, const float *a1Tf, cudaStream_t st) {
    const long long n = (long long)t->nk * t->nf * t->nf;
    const int grid = (int)std::min<long long>((n + 255) / 256, 4096);
    k_hs_fill<double><<<grid, 256, 0, st>>>(n, t->sidx, a1T, t->a1s64);
    k_hs_fill<float><<<grid, 256, 0, st>>>(n, t->sidx, a1Tf, t->a1s32);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

void hs_tables_free(HsTables *t) {
    cudaFree(t->srow);
    cudaFree(t->sidx);
    cudaFree(t->pp);
    cudaFree(t->pull);
    cudaFree(t->a1s64);
    cudaFree(t->a1s32);
    *t = HsTables();
}

size_t hs_smem_bytes(int npair, size_t w) { return (size_t)npair * kPairCols * w; }

int hs_block_cols(const HsTables &t, int len, size_t w) {
    const int full = (len + kPairCols - 1) / kPairCols * kPairCols;
    const size_t per_col = (size_t)t.nk * t.nf * w;
    const int cb = (int)std::min<size_t>(full, kPairEBytes / per_col / kPairCols * kPairCols);
    return std::max(cb, kPairCols);
}

// Y = the singles of rows x len matrix x (Y overwritten), jc [pair][column]
// the Coulomb parts, through E blocks of hs_block_cols columns.
template <typename T>
jci_status hs_launch(const HsTables &t, int len, int npair, const T *jc, const T *x, T *y,
                     const int *skip, T *E, int device, cudaStream_t st) {
    HsArgs<T> a;
    a.nk = t.nk; a.nf = t.nf; a.len = len; a.npair = npair;
    a.srow = t.srow; a.pp = t.pp; a.jc = jc; a.skip = skip;
    if constexpr (sizeof(T) == 8) a.a1s = t.a1s64;
    else a.a1s = t.a1s32;
    PairArgs<T> pa{};
    pa.nk = t.nk; pa.np = t.nf; pa.nt = t.nt; pa.rows = t.rows; pa.len = len;
    pa.pull = t.pull; pa.skip = skip;
    const size_t smem = hs_smem_bytes(npair, sizeof(T));
    int optin = 0;
    JCI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    if (smem > (size_t)optin) return JCI_ERR_SPACE;
    JCI_CUDA(smem_optin(k_hsingles_product<T>));
    const int cb = hs_block_cols(t, len, sizeof(T));
    const size_t psmem = (size_t)kPullRows * t.nt * sizeof(int);
    for (int c0 = 0; c0 < len; c0 += cb) {
        const int w = std::min(cb, len - c0);
        dim3 g1((t.nk + kHsPerCta - 1) / kHsPerCta, (w + kPairCols - 1) / kPairCols);
        k_hsingles_product<T><<<g1, 256, smem, st>>>(a, x, E, c0, cb);
        dim3 g2((t.rows + kPullRows - 1) / kPullRows, (w + kPairThreads - 1) / kPairThreads);
        k_pairs_pull<T><<<g2, kPairThreads, psmem, st>>>(pa, E, x, y, nullptr, 0, c0, cb);
    }
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

template jci_status hs_launch<double>(const HsTables &, int, int, const double *, const double *,
                                      double *, const int *, double *, int, cudaStream_t);
template jci_status hs_launch<float>(const HsTables &, int, int, const float *, const float *,
                                     float *, const int *, float *, int, cudaStream_t);

}  // namespace jci
