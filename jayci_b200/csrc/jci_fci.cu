// jci_fci.cu -- sigma = H c for spaces with one electron-occupation group
// per spin (FCI, CAS, and DOCC+ACTV with xlevel 0).
//
// With one group every alpha string pairs with every beta string, so the
// CI vector is an Nalpha x Nbeta row-major matrix (det = p * Nbeta + q,
// pdavidson.c:4757 with a single (p,q) pair), every string has the same
// number of singles / doubles, and the excitation tables can be stored
// transposed ([excitation][string]) so that the threads of a CTA, which own
// consecutive beta strings, read them coalesced.
//
// Kernel layout: one CTA per alpha string Ia computes the whole row
// sigma(Ia, :) in registers (each thread owns Nbeta / blockDim columns):
//   1. the CTA's own row c(Ia, :) is staged in shared memory; beta singles
//      and beta doubles gather from it (hmatels_1x / hmatels_2xaa on the
//      beta string, action_util.c:210,237);
//   2. alpha singles Ja are processed R rows at a time: rows c(Ja, :) and
//      the integral rows phase_a * (pa|.) are staged in shared memory; each
//      column applies the alpha single (same beta string, hmatels_1x) and
//      every beta single of its string against each staged row
//      (hmatels_2xab, action_util.c:250), so one load of a beta excitation
//      entry serves R rows;
//   3. alpha doubles stream rows c(Ja, :) straight from global memory
//      (coalesced, L2-resident for the sizes that fit).
// Each sigma element is written once (gather form): no atomics, and the
// result is bitwise reproducible run to run.
#include <algorithm>
#include <cstdio>
#include <cuda_pipeline.h>

#include <mutex>
#include <vector>

#include "jci_kernels.cuh"

namespace jci {

template <typename T>
struct FciSpin {
    T *a1T = nullptr;     // [single][string] one-body part, no phase
    T *joccT = nullptr;   // [pair][string] sum_{m in string} (mm|pair)
    T *dblH = nullptr;    // [double][string] value with phase
};

struct FciTables {
    int na = 0, nb = 0, sa = 0, sb = 0, da = 0, db = 0, npair = 0, nelb = 0;
    int *dblJ[2] = {nullptr, nullptr};   // [double][string] target string
    FciSpin<double> d[2];
    FciSpin<float> f[2];
    size_t smem_max = 0;
    int tuned_nt[2] = {0, 0}, tuned_R[2] = {0, 0};  // per precision (autotuned)
    int tuned_mode[2] = {0, 0}, tuned_B[2] = {1, 1};
    float tuned_ms[2] = {0.f, 0.f};
    int mix_grid[2] = {0, 0};      // resident CTAs of k_sigma_mixed
    int mix_occ[2] = {1, 1}, nsm = 0;
    void *tbuf[2] = {nullptr, nullptr};  // per-CTA product panels
    void *sbuf[2] = {nullptr, nullptr};  // streaming plan: C^T and the beta part (2 N)
    uint32_t *sortB = nullptr;     // [Ib][f] beta singles sorted by target
    AbTables ab[2];                // fused product's entry lists, 8 / 16 column threads
    GroupTables grp[2];            // same-spin doubles by string groups, per spin
    int *tc_status = nullptr;      // set by a product kernel whose bounded wait expired
                                   // (tcgen05 product, row-shared panels)
    AbTables abk;                  // per-block lists of the column-blocked panel product
    void *tbufk[2] = {nullptr, nullptr};  // its per-CTA scratch blocks
    int mixk_grid[2] = {0, 0};
    void *wbuf[2] = {nullptr, nullptr};   // row-shared panels of the queued product
    void *wctl[2] = {nullptr, nullptr};   // and its queue counters (WaveCtl)
    int wave_expire = 0;           // test hook: the next such launch skips work (see below)
    // compact product panel: per chunk and panel row the needed columns and
    // the first position, the gather's entry positions per beta string
    uint64_t *cp_mask = nullptr;
    int *cp_base = nullptr, *cp_gidx = nullptr;
    long long cp_len = 0;
    int cp_ent = 0, cp_state = 0;  // cp_state 0 not built, 1 built, -1 not possible
    PairTables prs[2];             // same-spin doubles through hole strings, per spin
    int prs_state = 0;             // 0 not built, 1 built, -1 not possible for this space
    HsTables hst;                  // beta singles through hole strings
    int hs_state = 0;              // as prs_state
    void *hbuf[2] = {nullptr, nullptr};  // their E blocks, per precision
    size_t hbytes[2] = {0, 0};
    void *pbuf[2] = {nullptr, nullptr};  // their E blocks, per precision
    size_t pbytes[2] = {0, 0};
};

bool fci_supported(const jci_space *s) {
    const DeviceState *d = s->dev;
    if (!d || !d->single_group || !d->fci) return false;
    return d->fci->smem_max > 0;
}

jci_status fci_arm_wait_expiry(jci_space *s) {
    if (!s->dev || !s->dev->fci) return JCI_ERR_STATE;
    s->dev->fci->wave_expire = 1;
    return JCI_OK;
}

jci_status fci_wait_status(jci_space *s) {
    const DeviceState *d = s->dev;
    if (!d || !d->fci || !d->fci->tc_status) return JCI_OK;
    int flag = 0;
    JCI_CUDA(cudaMemcpy(&flag, d->fci->tc_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (!flag) return JCI_OK;
    JCI_CUDA(cudaMemset(d->fci->tc_status, 0, sizeof(int)));
    return JCI_ERR_TIMEOUT;
}

void fci_free(DeviceState *d) {
    FciTables *f = d->fci;
    if (!f) return;
    for (int s = 0; s < 2; s++) {
        cudaFree(f->dblJ[s]);
        cudaFree(f->d[s].a1T); cudaFree(f->d[s].joccT); cudaFree(f->d[s].dblH);
        cudaFree(f->f[s].a1T); cudaFree(f->f[s].joccT); cudaFree(f->f[s].dblH);
        cudaFree(f->tbuf[s]);
        cudaFree(f->sbuf[s]);
    }
    cudaFree(f->sortB);
    cudaFree(f->tc_status);
    cudaFree(f->tbufk[0]);
    cudaFree(f->tbufk[1]);
    for (int p = 0; p < 2; p++) {
        cudaFree(f->wbuf[p]);
        cudaFree(f->wctl[p]);
    }
    ab_tables_free(&f->abk);
    ab_tables_free(&f->ab[0]);
    ab_tables_free(&f->ab[1]);
    group_tables_free(&f->grp[0]);
    group_tables_free(&f->grp[1]);
    pair_tables_free(&f->prs[0]);
    pair_tables_free(&f->prs[1]);
    hs_tables_free(&f->hst);
    cudaFree(f->hbuf[0]);
    cudaFree(f->hbuf[1]);
    cudaFree(f->cp_mask);
    cudaFree(f->cp_base);
    cudaFree(f->cp_gidx);
    cudaFree(f->pbuf[0]);
    cudaFree(f->pbuf[1]);
    delete f;
    d->fci = nullptr;
}

// ---- table construction -----------------------------------------------

__global__ void k_fci_tables(int nstr, int nelec, int ns, int nd, int npair,
                             const int *__restrict__ istr, const uint2 *__restrict__ doub,
                             const double *__restrict__ a1, const double *__restrict__ m2,
                             double *a1T, float *a1Tf, double *joccT, float *joccTf,
                             int *dblJ, double *dblH, float *dblHf) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nstr) return;
    for (int e = 0; e < ns; e++) {
        double v = a1[(long long)s * ns + e];
        a1T[(long long)e * nstr + s] = v;
        a1Tf[(long long)e * nstr + s] = (float)v;
    }
    const int *o = istr + (long long)s * nelec;
    for (int p = 0; p < npair; p++) {
        double v = 0.0;
        for (int k = 0; k < nelec; k++) v += m2[eri_index(pair_index(o[k], o[k]), p)];
        joccT[(long long)p * nstr + s] = v;
        joccTf[(long long)p * nstr + s] = (float)v;
    }
    for (int e = 0; e < nd; e++) {
        uint2 x = doub[(long long)s * nd + e];
        int i0 = x.y & 0xff, f0 = (x.y >> 8) & 0xff, i1 = (x.y >> 16) & 0xff, f1 = x.y >> 24;
        double h = m2[eri_index(pair_index(i0, f0), pair_index(i1, f1))] -
                   m2[eri_index(pair_index(i0, f1), pair_index(i1, f0))];
        if (x.x >> 31) h = -h;
        dblJ[(long long)e * nstr + s] = (int)(x.x & 0x3fffffffu);
        dblH[(long long)e * nstr + s] = h;
        dblHf[(long long)e * nstr + s] = (float)h;
    }
}

template <typename T>
struct FciArgs {
    int na, nb, sa, sb, da, db, npair, R;
    int do_as;                    // 0: alpha singles are left to k_sigma_mixed
    const uint32_t *fsA, *fsB;    // [single][string] target | sign << 31
    const uint16_t *fpA, *fpB;    // [single][string] pair index
    const T *a1A, *a1B;           // [single][string]
    const T *jA, *jB;             // [pair][string]
    const int *dJA, *dJB;         // [double][string]
    const T *dHA, *dHB;
    const T *hd;                  // <i|H|i>
    const T *m2;                  // packed (pq|rs)
    const int *skip;              // DeviceState::sigma_skip
};

template <typename T>
__device__ __forceinline__ T flip(T w, uint32_t neg) {
    return neg ? -w : w;
}

template <typename T, int ITEMS>
__global__ void __launch_bounds__(ITEMS <= 2 ? 1024 : 512)
    k_sigma_fci(FciArgs<T> a, const T *__restrict__ V, T *__restrict__ S) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *rows = reinterpret_cast<T *>(smem_raw);         // (1 + R) x nb
    T *vrow = rows + (size_t)(1 + a.R) * a.nb;         // R x npair
    T *jrow = vrow + (size_t)a.R * a.npair;            // npair
    T *coef = jrow + a.npair;                          // R
    int *pas = reinterpret_cast<int *>(coef + a.R);    // R pair of alpha single
    uint32_t *sgn = reinterpret_cast<uint32_t *>(pas + a.R);  // R
    const int nb = a.nb, tid = threadIdx.x, nt = blockDim.x;
    const int Ia = blockIdx.x;
    const T *crow = V + (long long)Ia * nb;
    for (int i = tid; i < nb; i += nt) rows[i] = crow[i];
    for (int p = tid; p < a.npair; p += nt) jrow[p] = a.jA[(long long)p * a.na + Ia];
    __syncthreads();

    // excitation index outer, the thread's ITEMS columns inner (unrolled):
    // ITEMS independent table loads in flight per excitation
    T acc[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        int Ib = tid + it * nt;
        acc[it] = Ib < nb ? a.hd[(long long)Ia * nb + Ib] * rows[Ib] : T(0);
    }
    // beta singles within the row (hmatels_1x with alpha as the other string)
    for (int f = 0; f < a.sb; f++) {
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib >= nb) continue;
            long long o = (long long)f * nb + Ib;
            uint32_t e = a.fsB[o];
            T h = a.a1B[o] + jrow[a.fpB[o]];
            acc[it] += flip(h, e >> 31) * rows[e & 0x3fffffffu];
        }
    }
    // beta doubles within the row
    for (int f = 0; f < a.db; f++) {
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib >= nb) continue;
            long long o = (long long)f * nb + Ib;
            acc[it] += a.dHB[o] * rows[a.dJB[o]];
        }
    }

    // alpha singles (with alpha x beta doubles), R staged rows at a time
    for (int e0 = 0; a.do_as && e0 < a.sa; e0 += a.R) {
        const int nr = min(a.R, a.sa - e0);
        __syncthreads();
        if (tid < nr) {
            long long o = (long long)(e0 + tid) * a.na + Ia;
            uint32_t e = a.fsA[o];
            sgn[tid] = e >> 31;
            pas[tid] = a.fpA[o];
            coef[tid] = flip(a.a1A[o], e >> 31);
        }
        __syncthreads();
        for (int r = 0; r < nr; r++) {
            long long o = (long long)(e0 + r) * a.na + Ia;
            int Ja = (int)(a.fsA[o] & 0x3fffffffu);
            const T *src = V + (long long)Ja * nb;
            T *dst = rows + (size_t)(1 + r) * nb;
            for (int i = tid; i < nb; i += nt) dst[i] = src[i];
            int pa = pas[r];
            uint32_t sg = sgn[r];
            for (int p = tid; p < a.npair; p += nt)
                vrow[(size_t)r * a.npair + p] = flip(a.m2[eri_index(pa, p)], sg);
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib >= nb) continue;
            T x = acc[it];
#pragma unroll 4
            for (int r = 0; r < nr; r++) {
                T h = coef[r] + flip(a.jB[(long long)pas[r] * nb + Ib], sgn[r]);
                x += h * rows[(size_t)(1 + r) * nb + Ib];
            }
            acc[it] = x;
        }
        for (int f = 0; f < a.sb; f++) {
#pragma unroll
            for (int it = 0; it < ITEMS; it++) {
                int Ib = tid + it * nt;
                if (Ib >= nb) continue;
                long long o = (long long)f * nb + Ib;
                uint32_t e = a.fsB[o];
                int J = (int)(e & 0x3fffffffu), pr = a.fpB[o];
                uint32_t neg = e >> 31;
                const T *rr = rows + nb + J;
                const T *vv = vrow + pr;
                T x = T(0);
#pragma unroll 4
                for (int r = 0; r < nr; r++) x += vv[(size_t)r * a.npair] * rr[(size_t)r * nb];
                acc[it] += flip(x, neg);
            }
        }
    }

    // alpha doubles: rows streamed from global memory
#pragma unroll 2
    for (int f = 0; f < a.da; f++) {
        long long o = (long long)f * a.na + Ia;
        int Ja = a.dJA[o];
        T h = a.dHA[o];
        const T *src = V + (long long)Ja * nb;
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib < nb) acc[it] += h * src[Ib];
        }
    }
    T *dst = S + (long long)Ia * nb;
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        int Ib = tid + it * nt;
        if (Ib < nb) dst[Ib] = acc[it];
    }
}

// ---- alpha singles and alpha x beta doubles as a dense product ------------
//
// For one alpha string Ia with alpha singles j -> (Ja_j, phase s_j, pair p_j):
//   T[p][Jb] = sum_j A[p][j] c(Ja_j, Jb),   A[p][j] = s_j (p_j | p)
//   T[U][Jb] = sum_j s_j a1(Ia, j) c(Ja_j, Jb)            (row U = npair)
// then, for every beta string Ib,
//   sigma(Ia, Ib) += T[U][Ib] + sum_{m in Ib} T[(mm)][Ib]
//                  + sum_{beta singles Ib -> Jb, pair q, phase t} t T[q][Jb].
// The first two terms are the alpha single elements (hmatels_1x with the
// beta string's Coulomb sum sum_{m in Ib} (mm|p_j)); the last is
// hmatels_2xab summed over both strings' singles.  The product runs in FP64
// on the FP64 tensor cores (mma.sync m8n8k4, 8 x 8 tiles, k in steps of 4)
// and in FP32 on the FMA pipes (a 16x16 thread grid, each thread holding a
// TM x 4 register tile); T goes to a per-CTA scratch panel in global memory
// (L2-resident for the mid sizes) and is gathered back in a fixed order, so
// results stay bitwise reproducible.

constexpr int kMixThreads = 256;
constexpr int kMixCols = 64;  // 16 threads x 4 columns per chunk

template <typename T>
struct MixArgs {
    int na, nb, nbp, sa, sb, npair, mrows;
    const uint32_t *fsA, *fsB;
    const uint16_t *fpA, *fpB;
    const T *a1A;
    const T *m2;
    const uint64_t *occB;
    const int *skip;
    // compact panel (null: the full mrows x nbp panel): only the entries the
    // gather reads are stored, row after row; cmask[c][m] marks the needed
    // columns of chunk c in panel row m, cbase[c][m] is the position of the
    // first of them, gidx[e][Ib] the gather's entries of string Ib in its
    // summation order (phase in bit 31), gent of them per string
    const uint64_t *cmask = nullptr;
    const int *cbase = nullptr;
    const int *gidx = nullptr;
    int gent = 0;
    long long plen = 0;  // compact panel entries per alpha row
};

// Shared-memory layout of the panel product: A [K4][AS] (alpha singles x
// panel rows), B [NB][K4][BS] (alpha singles x 64 columns), jl [K].  FP64
// runs the product on the FP64 tensor cores (mma.sync m8n8k4): K is padded
// to a multiple of 4 with zero rows, and A and B rows are padded by 4
// doubles so that a warp's fragment loads (rows k..k+3, 8 consecutive
// elements each) fall in distinct banks.  FP32 keeps the unpadded layout of
// its FMA form.
__host__ __device__ constexpr int mix_k4(int K, int w) { return w == 8 ? (K + 3) & ~3 : K; }
__host__ __device__ constexpr int mix_as(int TM, int w) { return 16 * TM + (w == 8 ? 4 : 0); }
__host__ __device__ constexpr int mix_bs(int w) { return kMixCols + (w == 8 ? 4 : 0); }

__device__ __forceinline__ void mix_dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// A and jl of alpha string Ia: A[j][m] = s_j (p_j | m) for the pairs m,
// s_j a1(Ia, j) in row U = npair, zero in the padding.
template <typename T, int TM>
__device__ __forceinline__ void mix_build_a(const MixArgs<T> &a, int Ia, T *As, int *jl) {
    constexpr int MP = 16 * TM, AS = mix_as(TM, sizeof(T));
    const int K = a.sa, K4 = mix_k4(K, sizeof(T));
    for (int idx = threadIdx.x; idx < K4 * MP; idx += kMixThreads) {
        const int j = idx / MP, m = idx - j * MP;
        T v = T(0);
        if (j < K) {
            const long long o = (long long)j * a.na + Ia;
            const uint32_t e = a.fsA[o];
            if (m < a.npair) v = a.m2[eri_index(a.fpA[o], m)];
            else if (m == a.npair) v = a.a1A[o];
            v = flip(v, e >> 31);
            if (m == 0) jl[j] = (int)(e & 0x3fffffffu);
        }
        As[j * AS + m] = v;
    }
}

// B chunk c: the 64 columns c*64.. of the rows jl of C (cp.async), zero past
// the last column and in the padding rows; one commit group.
template <typename T>
__device__ __forceinline__ void mix_stage(const MixArgs<T> &a, const T *__restrict__ V,
                                          const int *jl, int c, T *buf) {
    constexpr int BS = mix_bs(sizeof(T));
    const int K = a.sa, K4 = mix_k4(K, sizeof(T));
    const int c0 = c * kMixCols;
    for (int idx = threadIdx.x; idx < K4 * kMixCols; idx += kMixThreads) {
        const int j = idx >> 6, cc = idx & 63, col = c0 + cc;
        T *dst = buf + j * BS + cc;
        if (j < K && col < a.nb)
            __pipeline_memcpy_async(dst, V + (long long)jl[j] * a.nb + col, sizeof(T));
        else
            *dst = T(0);
    }
    __pipeline_commit();
}

// T[m][c0 + col] = sum_j A[j][m] B[j][col] for the panel rows m < mrows of
// one 64-column chunk, into the panel row stride nbp.  FP64: warp w owns
// columns 16 (w & 3) .. + 15 and panel rows 8 TM (w >> 2) .. + 8 TM - 1 as
// 2 x TM tiles of 8 x 8, accumulated over k in steps of 4 by mma.sync.
// FP32: the 16 x 16 thread grid, each thread a TM x 4 register tile.
// Position of panel entry (m, chunk column cc) in the compact panel, or -1
// when the gather never reads it (cm, cb: the chunk's masks and bases).
__device__ __forceinline__ int mix_cpos(const uint64_t *cm, const int *cb, int m, int cc) {
    const uint64_t w = cm[m];
    if (!((w >> cc) & 1)) return -1;
    return cb[m] + __popcll(w & ((1ull << cc) - 1));
}

template <typename T, int TM>
__device__ __forceinline__ void mix_product(const MixArgs<T> &a, const T *As, const T *Bc,
                                            T *Tb, int c0, const uint64_t *cm = nullptr,
                                            const int *cb = nullptr) {
    if constexpr (sizeof(T) == 8) {
        constexpr int AS = mix_as(TM, 8), BS = mix_bs(8);
        const int K4 = mix_k4(a.sa, 8);
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
        const int wn = warp & 3, wm = warp >> 2;
        double acc[TM][2][2];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int n = 0; n < 2; n++) acc[i][n][0] = acc[i][n][1] = 0.0;
        const double *ap = As + t * AS + 8 * TM * wm + g;
        const double *bp = Bc + t * BS + 16 * wn + g;
#pragma unroll 2
        for (int k0 = 0; k0 < K4; k0 += 4) {
            const double b0 = bp[k0 * BS], b1 = bp[k0 * BS + 8];
#pragma unroll
            for (int i = 0; i < TM; i++) {
                const double av = ap[k0 * AS + 8 * i];
                mix_dmma(acc[i][0], av, b0);
                mix_dmma(acc[i][1], av, b1);
            }
        }
        // accumulator layout: lane holds row g, columns 2t and 2t+1 of a tile
#pragma unroll
        for (int i = 0; i < TM; i++) {
            const int m = 8 * (TM * wm + i) + g;
            if (m < a.mrows) {
#pragma unroll
                for (int n = 0; n < 2; n++) {
                    const int cc = 16 * wn + 8 * n + 2 * t;
                    if (cm) {
#pragma unroll
                        for (int e = 0; e < 2; e++) {
                            const int q = mix_cpos(cm, cb, m, cc + e);
                            if (q >= 0) Tb[q] = acc[i][n][e];
                        }
                    } else {
                        *reinterpret_cast<double2 *>(Tb + (size_t)m * a.nbp + c0 + cc) =
                            make_double2(acc[i][n][0], acc[i][n][1]);
                    }
                }
            }
        }
    } else {
        constexpr int MP = 16 * TM;
        const int K = a.sa, tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
        T acc[TM][4];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][q] = T(0);
#pragma unroll 4
        for (int k = 0; k < K; k++) {
            // thread tx owns columns tx, tx+16, tx+32, tx+48: a warp reads
            // 16 consecutive words per load (no bank conflicts)
            const T *br = Bc + k * kMixCols + tx;
            T b0 = br[0], b1 = br[16], b2 = br[32], b3 = br[48];
            const T *ar = As + k * MP + ty * TM;
#pragma unroll
            for (int i = 0; i < TM; i++) {
                T av = ar[i];
                acc[i][0] = fma(av, b0, acc[i][0]);
                acc[i][1] = fma(av, b1, acc[i][1]);
                acc[i][2] = fma(av, b2, acc[i][2]);
                acc[i][3] = fma(av, b3, acc[i][3]);
            }
        }
#pragma unroll
        for (int i = 0; i < TM; i++) {
            int m = ty * TM + i;
            if (m < a.mrows) {
                if (cm) {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const int p = mix_cpos(cm, cb, m, tx + 16 * q);
                        if (p >= 0) Tb[p] = acc[i][q];
                    }
                } else {
                    T *dst = Tb + (size_t)m * a.nbp + c0 + tx;
#pragma unroll
                    for (int q = 0; q < 4; q++) dst[16 * q] = acc[i][q];
                }
            }
        }
    }
}

// NB = 2: B chunks double-buffered (chunk c+1 copied while chunk c
// multiplies); NB = 1: one buffer, so that two CTAs fit an SM where the
// double-buffered form fits one (the other CTA's product then covers this
// CTA's copies and gather).
template <typename T, int TM, int NB = 2>
__global__ void __launch_bounds__(kMixThreads)
    k_sigma_mixed(MixArgs<T> a, const T *__restrict__ V, T *__restrict__ S, T *__restrict__ Tbuf) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K4 = mix_k4(a.sa, sizeof(T));
    T *As = reinterpret_cast<T *>(smem_raw);                          // [K4][AS]
    T *Bs = As + (size_t)K4 * mix_as(TM, sizeof(T));                  // [NB][K4][BS]
    int *jl = reinterpret_cast<int *>(Bs + NB * (size_t)K4 * mix_bs(sizeof(T)));  // [K]
    // compact panel: the chunk's masks and bases, [mrows] each
    uint64_t *cm = reinterpret_cast<uint64_t *>(jl + ((a.sa + 1) & ~1));
    int *cb = reinterpret_cast<int *>(cm + a.mrows);
    const bool cp = a.cmask != nullptr;
    const size_t bsz = (size_t)K4 * mix_bs(sizeof(T));
    const int tid = threadIdx.x;
    T *Tb = Tbuf + (size_t)blockIdx.x * (cp ? (size_t)a.plen : (size_t)a.mrows * a.nbp);
    const int nchunk = a.nbp / kMixCols;
    for (int Ia = blockIdx.x; Ia < a.na; Ia += gridDim.x) {
        __syncthreads();
        mix_build_a<T, TM>(a, Ia, As, jl);
        __syncthreads();
        mix_stage<T>(a, V, jl, 0, Bs);
        for (int ci = 0; ci < nchunk; ci++) {
            T *Bc = Bs + (NB == 2 ? (ci & 1) : 0) * bsz;
            if (NB == 2 && ci + 1 < nchunk) {
                mix_stage<T>(a, V, jl, ci + 1, Bs + ((ci + 1) & 1) * bsz);
                __pipeline_wait_prior(1);
            } else {
                __pipeline_wait_prior(0);
            }
            if (cp)
                for (int m = tid; m < a.mrows; m += kMixThreads) {
                    cm[m] = a.cmask[(size_t)ci * a.mrows + m];
                    cb[m] = a.cbase[(size_t)ci * a.mrows + m];
                }
            __syncthreads();
            mix_product<T, TM>(a, As, Bc, Tb, ci * kMixCols, cp ? cm : nullptr, cb);
            __syncthreads();
            if (NB == 1 && ci + 1 < nchunk) mix_stage<T>(a, V, jl, ci + 1, Bs);
        }
        // gather: every column of the row owned by one thread, fixed order.
        // The panel reads are random (DRAM once the panels outgrow L2); the
        // singles loop takes its indices 8 at a time so that 8 panel reads
        // are in flight per thread, and adds them in list order.
        T *srow = S + (long long)Ia * a.nb;
        if (cp) {
            // the same terms in the same order, at their compact positions
            for (int Ib = tid; Ib < a.nb; Ib += kMixThreads) {
                const int *gi = a.gidx + Ib;
                T x = Tb[gi[0]];
                int e = 1;
                for (; e + 8 <= a.gent; e += 8) {
                    T t[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        const int g = gi[(size_t)(e + u) * a.nb];
                        t[u] = flip(Tb[g & 0x7fffffff], (uint32_t)g >> 31);
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) x += t[u];
                }
                for (; e < a.gent; e++) {
                    const int g = gi[(size_t)e * a.nb];
                    x += flip(Tb[g & 0x7fffffff], (uint32_t)g >> 31);
                }
                srow[Ib] += x;
            }
            continue;
        }
        const T *TU = Tb + (size_t)a.npair * a.nbp;
        for (int Ib = tid; Ib < a.nb; Ib += kMixThreads) {
            T x = TU[Ib];
            uint64_t oc = a.occB[Ib];
            while (oc) {
                int m = __ffsll((long long)oc);  // 1-based orbital
                oc &= oc - 1;
                x += Tb[(size_t)(m * (m + 1) / 2 - 1) * a.nbp + Ib];
            }
            int f = 0;
            for (; f + 8 <= a.sb; f += 8) {
                T t[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    const long long o = (long long)(f + u) * a.nb + Ib;
                    const uint32_t e = a.fsB[o];
                    t[u] = flip(Tb[(size_t)a.fpB[o] * a.nbp + (e & 0x3fffffffu)], e >> 31);
                }
#pragma unroll
                for (int u = 0; u < 8; u++) x += t[u];
            }
            for (; f < a.sb; f++) {
                long long o = (long long)f * a.nb + Ib;
                uint32_t e = a.fsB[o];
                x += flip(Tb[(size_t)a.fpB[o] * a.nbp + (e & 0x3fffffffu)], e >> 31);
            }
            srow[Ib] += x;
        }
    }
}

// ---- dense product through a column-blocked panel --------------------------
//
// The product of k_sigma_mixed with its panel cut into blocks of kMixBlock
// columns: the CTA forms T[:, block] (kMixBlock / 64 chunks, as above) in a
// scratch block of mrows x kMixBlock, then gathers the block's share of every
// beta string's terms -- the entries of the per-block lists (ab_tables_build
// with 4 tx = kMixBlock: the one-body row, the Coulomb rows and the singles
// whose target column lies in the block, in list order) -- and adds it to
// sigma(Ia, Ib) in place.  The scratch block (FCI(16,16): 137 x 256 x 8 B =
// 280 KB) and the sigma row stay in L2, where the whole-row panel (14 MB)
// spilled to DRAM and its gather read it at random.  Sums run block by
// block, then in list order: bitwise reproducible.
constexpr int kMixBlock = 256;

template <typename T>
struct MixBArgs {
    MixArgs<T> m;
    int offs;                 // offset row stride of the block lists
    const uint16_t *off;      // [block][offs]
    const uint32_t *base;     // [block + 1]
    const uint32_t *ent;      // col | row << 8 | phase << 31
};

template <typename T, int TM>
__global__ void __launch_bounds__(kMixThreads)
    k_sigma_mixed_blk(MixBArgs<T> ab, const T *__restrict__ V, T *__restrict__ S,
                      T *__restrict__ Tbuf) {
    const MixArgs<T> &a = ab.m;
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int MP = 16 * TM;
    constexpr int CPB = kMixBlock / kMixCols;  // chunks per block
    const int K = a.sa;
    T *As = reinterpret_cast<T *>(smem_raw);          // [K][MP]
    T *Bs = As + (size_t)K * MP;                      // [2][K][64]
    int *jl = reinterpret_cast<int *>(Bs + 2 * (size_t)K * kMixCols);  // [K]
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    T *Tb = Tbuf + (size_t)blockIdx.x * a.mrows * kMixBlock;
    const int nchunk = a.nbp / kMixCols;
    auto stage = [&](int c, T *buf) {
        const int c0 = c * kMixCols;
        for (int idx = tid; idx < K * kMixCols; idx += kMixThreads) {
            int j = idx >> 6, col = c0 + (idx & 63);
            if (col < a.nb)
                __pipeline_memcpy_async(buf + idx, V + (long long)jl[j] * a.nb + col, sizeof(T));
            else
                buf[idx] = T(0);
        }
        __pipeline_commit();
    };
    for (int Ia = blockIdx.x; Ia < a.na; Ia += gridDim.x) {
        __syncthreads();
        for (int idx = tid; idx < K * MP; idx += kMixThreads) {
            int j = idx / MP, m = idx - j * MP;
            long long o = (long long)j * a.na + Ia;
            uint32_t e = a.fsA[o];
            T v = T(0);
            if (m < a.npair) v = a.m2[eri_index(a.fpA[o], m)];
            else if (m == a.npair) v = a.a1A[o];
            As[idx] = flip(v, e >> 31);
            if (m == 0) jl[j] = (int)(e & 0x3fffffffu);
        }
        __syncthreads();
        T *srow = S + (long long)Ia * a.nb;
        stage(0, Bs);
        for (int ci = 0; ci < nchunk; ci++) {
            const int cb = ci % CPB;
            T *Bc = Bs + (size_t)(ci & 1) * K * kMixCols;
            if (ci + 1 < nchunk) {
                stage(ci + 1, Bs + (size_t)((ci + 1) & 1) * K * kMixCols);
                __pipeline_wait_prior(1);
            } else {
                __pipeline_wait_prior(0);
            }
            __syncthreads();
            T acc[TM][4];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[i][q] = T(0);
#pragma unroll 4
            for (int k = 0; k < K; k++) {
                const T *br = Bc + k * kMixCols + tx;
                T b0 = br[0], b1 = br[16], b2 = br[32], b3 = br[48];
                const T *ar = As + k * MP + ty * TM;
#pragma unroll
                for (int i = 0; i < TM; i++) {
                    T av = ar[i];
                    acc[i][0] = fma(av, b0, acc[i][0]);
                    acc[i][1] = fma(av, b1, acc[i][1]);
                    acc[i][2] = fma(av, b2, acc[i][2]);
                    acc[i][3] = fma(av, b3, acc[i][3]);
                }
            }
#pragma unroll
            for (int i = 0; i < TM; i++) {
                int m = ty * TM + i;
                if (m < a.mrows) {
                    T *dst = Tb + (size_t)m * kMixBlock + cb * kMixCols + tx;
#pragma unroll
                    for (int q = 0; q < 4; q++) dst[16 * q] = acc[i][q];
                }
            }
            if (cb == CPB - 1 || ci + 1 == nchunk) {
                // the block is complete: gather its terms into sigma(Ia, :)
                __syncthreads();
                const int blk = ci / CPB;
                const uint16_t *off = ab.off + (size_t)blk * ab.offs;
                const uint32_t *ent = ab.ent + ab.base[blk];
                for (int Ib = tid; Ib < a.nb; Ib += kMixThreads) {
                    const int k0 = off[Ib], k1 = off[Ib + 1];
                    if (k0 == k1) continue;
                    T x = T(0);
                    for (int k = k0; k < k1; k++) {
                        const uint32_t e = ent[k];
                        x += flip(Tb[(size_t)((e >> 8) & 0xffffu) * kMixBlock + (e & 0xffu)],
                                  e >> 31);
                    }
                    srow[Ib] += x;
                }
            }
            __syncthreads();
        }
    }
}

// ---- dense product through row panels shared by all CTAs -------------------
//
// The product of k_sigma_mixed with each alpha string's panel T (mrows x nbp)
// built by many CTAs at once and kept in L2, instead of one private panel
// per CTA (296 panels of 14 MB at FCI(16,16): written to and gathered back
// from DRAM at random).  The work is a queue of items claimed with one
// atomic counter:
//   step i:  the GEMM items of row i (kWaveChunks 64-column chunks of T each),
//            then the gather items of row i - kWaveLag (kMixThreads beta
//            strings each: the same sums as k_sigma_mixed's gather);
// row i's panel is buffer i % kWaveBufs.  A gather item waits until all GEMM
// items of its row are done; a GEMM item waits until all gather items of
// the row that used its buffer before are done.  Every wait is on an item
// that was claimed earlier (kWaveBufs > kWaveLag), by a CTA that is running,
// so the queue cannot stall on residency; waits are bounded (one second of
// global time), after which the kernel sets *status and returns.  Each T
// element and each sigma element is computed by one item in the order of
// k_sigma_mixed: the result is bitwise that of k_sigma_mixed.
constexpr int kWaveBufs = 4, kWaveLag = 2, kWaveChunks = 4;

struct WaveCtl {
    int next;                    // next item to claim
    int err;                     // a bounded wait expired
    int gemm_done[kWaveBufs];    // GEMM items finished per buffer (cumulative)
    int gather_done[kWaveBufs];  // gather items finished per buffer (cumulative)
};

__device__ __forceinline__ uint64_t wave_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Thread 0: wait until *cnt >= target; false after about one second or when
// another CTA has given up (ctl->err).
__device__ __forceinline__ bool wave_wait(const int *cnt, int target, WaveCtl *ctl) {
    const uint64_t t0 = wave_ns();
    for (long long it = 0;; it++) {
        int v;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
        if (v >= target) return true;
        if ((it & 63) == 63) {
            if (*(volatile int *)&ctl->err) return false;
            if (wave_ns() - t0 > 1000000000ull || it > (1ll << 28)) return false;
        }
        __nanosleep(64);
    }
}

template <typename T, int TM, int NB>
__global__ void __launch_bounds__(kMixThreads)
    k_sigma_wave(MixArgs<T> a, const T *__restrict__ V, T *__restrict__ S, T *__restrict__ Tw,
                 WaveCtl *ctl, int ngi, int nhi, int *status) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item, s_ok;
    const int K4 = mix_k4(a.sa, sizeof(T));
    T *As = reinterpret_cast<T *>(smem_raw);                          // [K4][AS]
    T *Bs = As + (size_t)K4 * mix_as(TM, sizeof(T));                  // [NB][K4][BS]
    int *jl = reinterpret_cast<int *>(Bs + NB * (size_t)K4 * mix_bs(sizeof(T)));  // [K]
    const size_t bsz = (size_t)K4 * mix_bs(sizeof(T));
    const int tid = threadIdx.x;
    const int nchunk = a.nbp / kMixCols;
    const size_t panel = (size_t)a.mrows * a.nbp;
    const int lag = min(kWaveLag, a.na), per = ngi + nhi;
    const long long pre = (long long)lag * ngi, mid = (long long)(a.na - lag) * per;
    const long long total = (long long)a.na * per;
    for (;;) {
        __syncthreads();  // the previous item is done with shared memory
        if (tid == 0) s_item = atomicAdd(&ctl->next, 1);
        __syncthreads();
        const long long q = s_item;
        if (q >= total) return;
        int row, sub;
        bool gemm;
        if (q < pre) {
            row = (int)(q / ngi); sub = (int)(q % ngi); gemm = true;
        } else if (q - pre < mid) {
            const long long r = q - pre;
            const int step = lag + (int)(r / per), k = (int)(r % per);
            gemm = k < ngi;
            row = gemm ? step : step - lag;
            sub = gemm ? k : k - ngi;
        } else {
            const long long r = q - pre - mid;
            row = a.na - lag + (int)(r / nhi); sub = (int)(r % nhi); gemm = false;
        }
        const int buf = row % kWaveBufs, gen = row / kWaveBufs;
        T *Tb = Tw + (size_t)buf * panel;
        if (tid == 0) {
            bool ok = gemm ? (gen == 0 || wave_wait(&ctl->gather_done[buf], gen * nhi, ctl))
                           : wave_wait(&ctl->gemm_done[buf], (gen + 1) * ngi, ctl);
            if (!ok) {
                atomicExch(&ctl->err, 1);
                if (status) atomicExch(status, 1);
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) return;
        if (gemm) {
            mix_build_a<T, TM>(a, row, As, jl);
            __syncthreads();
            const int c_lo = sub * kWaveChunks, c_hi = min(nchunk, c_lo + kWaveChunks);
            mix_stage<T>(a, V, jl, c_lo, Bs);
            for (int ci = c_lo; ci < c_hi; ci++) {
                T *Bc = Bs + (NB == 2 ? ((ci - c_lo) & 1) : 0) * bsz;
                if (NB == 2 && ci + 1 < c_hi) {
                    mix_stage<T>(a, V, jl, ci + 1, Bs + ((ci + 1 - c_lo) & 1) * bsz);
                    __pipeline_wait_prior(1);
                } else {
                    __pipeline_wait_prior(0);
                }
                __syncthreads();
                mix_product<T, TM>(a, As, Bc, Tb, ci * kMixCols);
                __syncthreads();
                if (NB == 1 && ci + 1 < c_hi) mix_stage<T>(a, V, jl, ci + 1, Bs);
            }
            // release (the pattern of a grid barrier): the CTA's panel stores,
            // then one thread's fence and count
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                atomicAdd(&ctl->gemm_done[buf], 1);
            }
        } else {
            const int Ia = row, Ib = sub * kMixThreads + tid;
            if (Ib < a.nb) {
                // panel reads from L2 (__ldcg): the buffer was rewritten by
                // other SMs since this SM last read it
                const T *TU = Tb + (size_t)a.npair * a.nbp;
                T x = __ldcg(TU + Ib);
                uint64_t oc = a.occB[Ib];
                while (oc) {
                    int m = __ffsll((long long)oc);
                    oc &= oc - 1;
                    x += __ldcg(Tb + (size_t)(m * (m + 1) / 2 - 1) * a.nbp + Ib);
                }
                int f = 0;
                for (; f + 8 <= a.sb; f += 8) {
                    T t[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) {
                        const long long o = (long long)(f + u) * a.nb + Ib;
                        const uint32_t e = a.fsB[o];
                        t[u] = flip(__ldcg(Tb + (size_t)a.fpB[o] * a.nbp + (e & 0x3fffffffu)),
                                    e >> 31);
                    }
#pragma unroll
                    for (int u = 0; u < 8; u++) x += t[u];
                }
                for (; f < a.sb; f++) {
                    long long o = (long long)f * a.nb + Ib;
                    uint32_t e = a.fsB[o];
                    x += flip(__ldcg(Tb + (size_t)a.fpB[o] * a.nbp + (e & 0x3fffffffu)), e >> 31);
                }
                S[(long long)Ia * a.nb + Ib] += x;
            }
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                atomicAdd(&ctl->gather_done[buf], 1);
            }
        }
    }
}

// ---- dense product without a global panel ---------------------------------
//
// Same product as k_sigma_mixed, but each 64-column chunk of T is kept in
// shared memory and consumed at once: every beta string Ib walks its singles
// sorted by target (sortB, J | pair << 16 | sign << 31) and adds the entries
// whose target falls in the current chunk; the one-body and Coulomb rows are
// added when the chunk holds Ib itself.  Per-string accumulators and walk
// positions live in shared memory, one owner thread per string, so the sums
// are taken in a fixed order (bitwise reproducible) and T never leaves the SM.

template <typename T>
struct Mix2Args {
    int na, nb, nbp, sa, sb, npair, mrows;
    const uint32_t *fsA;
    const uint16_t *fpA;
    const uint32_t *sortB;   // [Ib][f] sorted by target
    const T *a1A;
    const T *m2;
    const uint64_t *occB;
    const int *skip;
};

template <typename T, int TM>
__global__ void __launch_bounds__(kMixThreads)
    k_sigma_mixed2(Mix2Args<T> a, const T *__restrict__ V, T *__restrict__ S) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int MP = 16 * TM;
    const int K = a.sa, nb = a.nb;
    T *As = reinterpret_cast<T *>(smem_raw);          // [K][MP]
    T *Bs = As + (size_t)K * MP;                      // [2][K][64]
    T *Ts = Bs + 2 * (size_t)K * kMixCols;            // [mrows][64]
    T *accs = Ts + (size_t)a.mrows * kMixCols;        // [nb]
    int *jl = reinterpret_cast<int *>(accs + nb);     // [K]
    unsigned char *pos = reinterpret_cast<unsigned char *>(jl + K);  // [nb]
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int nchunk = a.nbp / kMixCols;
    auto stage = [&](int c, T *buf) {
        const int c0 = c * kMixCols;
        for (int idx = tid; idx < K * kMixCols; idx += kMixThreads) {
            int j = idx >> 6, col = c0 + (idx & 63);
            if (col < nb)
                __pipeline_memcpy_async(buf + idx, V + (long long)jl[j] * nb + col, sizeof(T));
            else
                buf[idx] = T(0);
        }
        __pipeline_commit();
    };
    for (int Ia = blockIdx.x; Ia < a.na; Ia += gridDim.x) {
        __syncthreads();
        for (int idx = tid; idx < K * MP; idx += kMixThreads) {
            int j = idx / MP, m = idx - j * MP;
            long long o = (long long)j * a.na + Ia;
            uint32_t e = a.fsA[o];
            T v = T(0);
            if (m < a.npair) v = a.m2[eri_index(a.fpA[o], m)];
            else if (m == a.npair) v = a.a1A[o];
            As[idx] = flip(v, e >> 31);
            if (m == 0) jl[j] = (int)(e & 0x3fffffffu);
        }
        for (int i = tid; i < nb; i += kMixThreads) {
            accs[i] = T(0);
            pos[i] = 0;
        }
        __syncthreads();
        stage(0, Bs);
        for (int ci = 0; ci < nchunk; ci++) {
            const int c0 = ci * kMixCols;
            T *Bc = Bs + (size_t)(ci & 1) * K * kMixCols;
            if (ci + 1 < nchunk) {
                stage(ci + 1, Bs + (size_t)((ci + 1) & 1) * K * kMixCols);
                __pipeline_wait_prior(1);
            } else {
                __pipeline_wait_prior(0);
            }
            __syncthreads();
            T acc[TM][4];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[i][q] = T(0);
#pragma unroll 4
            for (int k = 0; k < K; k++) {
                const T *br = Bc + k * kMixCols + tx;
                T b0 = br[0], b1 = br[16], b2 = br[32], b3 = br[48];
                const T *ar = As + k * MP + ty * TM;
#pragma unroll
                for (int i = 0; i < TM; i++) {
                    T av = ar[i];
                    acc[i][0] = fma(av, b0, acc[i][0]);
                    acc[i][1] = fma(av, b1, acc[i][1]);
                    acc[i][2] = fma(av, b2, acc[i][2]);
                    acc[i][3] = fma(av, b3, acc[i][3]);
                }
            }
#pragma unroll
            for (int i = 0; i < TM; i++) {
                int m = ty * TM + i;
                if (m < a.mrows) {
                    T *dst = Ts + (size_t)m * kMixCols + tx;
#pragma unroll
                    for (int q = 0; q < 4; q++) dst[16 * q] = acc[i][q];
                }
            }
            __syncthreads();
            const int c1 = c0 + kMixCols;
            for (int Ib = tid; Ib < nb; Ib += kMixThreads) {
                T x = accs[Ib];
                int p = pos[Ib];
                const uint32_t *lst = a.sortB + (size_t)Ib * a.sb;
                while (p < a.sb) {
                    uint32_t e = lst[p];
                    int J = (int)(e & 0xffffu);
                    if (J >= c1) break;
                    x += flip(Ts[(size_t)((e >> 16) & 0x7fffu) * kMixCols + (J - c0)], e >> 31);
                    p++;
                }
                if (Ib >= c0 && Ib < c1) {
                    const int col = Ib - c0;
                    x += Ts[(size_t)a.npair * kMixCols + col];
                    uint64_t oc = a.occB[Ib];
                    while (oc) {
                        int m = __ffsll((long long)oc);
                        oc &= oc - 1;
                        x += Ts[(size_t)(m * (m + 1) / 2 - 1) * kMixCols + col];
                    }
                }
                accs[Ib] = x;
                pos[Ib] = (unsigned char)p;
            }
            __syncthreads();
        }
        T *srow = S + (long long)Ia * nb;
        for (int Ib = tid; Ib < nb; Ib += kMixThreads) srow[Ib] += accs[Ib];
    }
}

static size_t mix2_smem(int K, int TM, int mrows, int nb, size_t w) {
    return (size_t)K * 16 * TM * w + 2 * (size_t)K * kMixCols * w + (size_t)mrows * kMixCols * w +
           (size_t)nb * w + (size_t)K * 4 + (size_t)nb + 64;
}

// ---- row kernel of the dense-product plan ---------------------------------
//
// RB consecutive alpha strings per CTA: the diagonal, the beta singles and
// beta doubles inside each row (gathered from the RB rows staged in shared
// memory, so one load of a beta excitation entry serves RB rows) and the
// alpha doubles (rows streamed from global memory).  The alpha singles are
// added by k_sigma_mixed afterwards.
//
// Loop order: the excitation index is the outer loop and the ITEMS columns
// of a thread the inner, unrolled one, so each warp has ITEMS independent
// table loads (and shared-memory gathers) in flight per excitation instead
// of one.  The alpha-double list of every row (target, value) is staged in
// shared memory first, so streaming a row c(Ja, :) waits on one global
// load, not two.

template <typename T, int ITEMS, int RB>
__global__ void __launch_bounds__(ITEMS * RB <= 4 ? 1024 : 512)
    k_sigma_rows(FciArgs<T> a, const T *__restrict__ V, T *__restrict__ S) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *rows = reinterpret_cast<T *>(smem_raw);   // RB x nb
    T *jrow = rows + (size_t)RB * a.nb;          // RB x npair
    T *dh = jrow + (size_t)RB * a.npair;         // RB x da  alpha-double values
    int *dj = reinterpret_cast<int *>(dh + (size_t)RB * a.da);  // RB x da targets
    const int nb = a.nb, tid = threadIdx.x, nt = blockDim.x;
    const int Ia0 = blockIdx.x * RB;
    const int nr = min(RB, a.na - Ia0);
    for (int r = 0; r < nr; r++) {
        const T *crow = V + (long long)(Ia0 + r) * nb;
        for (int i = tid; i < nb; i += nt) rows[(size_t)r * nb + i] = crow[i];
        for (int p = tid; p < a.npair; p += nt)
            jrow[(size_t)r * a.npair + p] = a.jA[(long long)p * a.na + Ia0 + r];
        for (int f = tid; f < a.da; f += nt) {
            long long o = (long long)f * a.na + Ia0 + r;
            dh[(size_t)r * a.da + f] = a.dHA[o];
            dj[(size_t)r * a.da + f] = a.dJA[o];
        }
    }
    __syncthreads();
    T acc[ITEMS][RB];
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        int Ib = tid + it * nt;
#pragma unroll
        for (int r = 0; r < RB; r++)
            acc[it][r] = Ib < nb && r < nr
                             ? a.hd[(long long)(Ia0 + r) * nb + Ib] * rows[(size_t)r * nb + Ib]
                             : T(0);
    }
    // beta singles within the rows (hmatels_1x with the alpha string's
    // Coulomb row jrow)
    for (int f = 0; f < a.sb; f++) {
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib >= nb) continue;
            long long o = (long long)f * nb + Ib;
            uint32_t e = a.fsB[o];
            T h = a.a1B[o];
            int J = (int)(e & 0x3fffffffu), pr = a.fpB[o];
            uint32_t neg = e >> 31;
#pragma unroll
            for (int r = 0; r < RB; r++)
                acc[it][r] += flip(h + jrow[(size_t)r * a.npair + pr], neg) *
                              rows[(size_t)r * nb + J];
        }
    }
    // beta doubles within the rows
    for (int f = 0; f < a.db; f++) {
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib >= nb) continue;
            long long o = (long long)f * nb + Ib;
            T h = a.dHB[o];
            int J = a.dJB[o];
#pragma unroll
            for (int r = 0; r < RB; r++) acc[it][r] += h * rows[(size_t)r * nb + J];
        }
    }
    // alpha doubles of each row: coefficient uniform over the CTA
#pragma unroll
    for (int r = 0; r < RB; r++) {
        if (r >= nr) break;
#pragma unroll 2
        for (int f = 0; f < a.da; f++) {
            const T h = dh[(size_t)r * a.da + f];
            const T *src = V + (long long)dj[(size_t)r * a.da + f] * nb;
#pragma unroll
            for (int it = 0; it < ITEMS; it++) {
                int Ib = tid + it * nt;
                if (Ib < nb) acc[it][r] += h * src[Ib];
            }
        }
    }
#pragma unroll
    for (int r = 0; r < RB; r++) {
        if (r >= nr) break;
        T *dst = S + (long long)(Ia0 + r) * nb;
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int Ib = tid + it * nt;
            if (Ib < nb) dst[Ib] = acc[it][r];
        }
    }
}

// ---- streaming plans (modes 3, 4; the beta singles of modes 6, 7) ----------
//
// Every term whose coefficient is the same for a whole row runs as row
// streams: the diagonal and the alpha doubles on C (rows Ia), and the beta
// singles and doubles on the transpose C^T (rows Ib), where they play the
// role the alpha excitations play on C.  A CTA loads its output row's
// excitation list once into shared memory; each excitation then reads one
// whole source row, coalesced, from L2 (the vector stays resident), and no
// per-element excitation table is read.  The beta part is added back to
// sigma with a tiled transpose; the alpha singles and alpha x beta doubles
// come from a product kernel (k_sigma_mixed or k_sigma_ab).  Modes 6 and 7
// keep only the beta singles here and take the doubles by string groups
// (jci_fci_group.cu).  Every sigma element is still summed in a fixed
// order.

constexpr int kTile = 32;

// dst[c][r] = src[r][c]  (src rows x cols); 32 x 32 tiles, block (32, 8)
template <typename T>
__global__ void k_transpose(const T *__restrict__ src, int rows, int cols, T *__restrict__ dst,
                            const int *skip) {
    if (skip && *skip) return;
    __shared__ T tile[kTile][kTile + 1];
    const int c0 = blockIdx.x * kTile, r0 = blockIdx.y * kTile;
    for (int j = threadIdx.y; j < kTile; j += 8) {
        int r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[j][threadIdx.x] = src[(long long)r * cols + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kTile; j += 8) {
        int c = c0 + j, r = r0 + threadIdx.x;
        if (c < cols && r < rows) dst[(long long)c * rows + r] = tile[threadIdx.x][j];
    }
}

// dst[r][c] += src[c][r]  (dst rows x cols, src cols x rows)
template <typename T>
__global__ void k_transpose_add(T *__restrict__ dst, int rows, int cols,
                                const T *__restrict__ src, const int *skip) {
    if (skip && *skip) return;
    __shared__ T tile[kTile][kTile + 1];
    const int c0 = blockIdx.x * kTile, r0 = blockIdx.y * kTile;
    for (int j = threadIdx.y; j < kTile; j += 8) {
        int sc = c0 + j, sr = r0 + threadIdx.x;
        if (sc < cols && sr < rows) tile[j][threadIdx.x] = src[(long long)sc * rows + sr];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kTile; j += 8) {
        int r = r0 + j, c = c0 + threadIdx.x;
        if (r < rows && c < cols) dst[(long long)r * cols + c] += tile[threadIdx.x][j];
    }
}

template <typename T>
struct StreamArgs {
    int rows, len;                // output rows x row length
    int nd, ns;                   // doubles / singles of every row (ns = 0: none)
    const int *dJ;                // [double][row] source row
    const T *dH;                  // [double][row] value with phase
    const uint32_t *fs;           // [single][row] source row | sign << 31
    const uint16_t *fp;           // [single][row] pair index
    const T *a1;                  // [single][row] one-body part
    const T *jc;                  // [pair][column] Coulomb part of a single
    const T *hd;                  // [row][column] diagonal, or null
    const int *skip;
};

// Y[row][i] = hd[row][i] X[row][i] + sum_f dH_f X[dJ_f][i]
//           + sum_f sign_f (a1_f + jc[pair_f][i]) X[target_f][i]
// for the columns i of segment blockIdx.y (seg columns each), so that a
// thread holds at most ITEMS <= 16 accumulators however long the rows are.
template <typename T, int ITEMS>
__global__ void __launch_bounds__(ITEMS <= 8 ? 1024 : 512)
    k_sigma_stream(StreamArgs<T> a, int seg, const T *__restrict__ X, T *__restrict__ Y) {
    if (a.skip && *a.skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *dh = reinterpret_cast<T *>(smem_raw);               // nd
    T *sh = dh + a.nd;                                     // ns
    int *dj = reinterpret_cast<int *>(sh + a.ns);          // nd
    uint32_t *se = reinterpret_cast<uint32_t *>(dj + a.nd);  // ns
    int *sp = reinterpret_cast<int *>(se + a.ns);          // ns
    const int row = blockIdx.x, tid = threadIdx.x, nt = blockDim.x, len = a.len;
    const int c0 = blockIdx.y * seg, c1 = min(len, c0 + seg);
    for (int f = tid; f < a.nd; f += nt) {
        long long o = (long long)f * a.rows + row;
        dh[f] = a.dH[o];
        dj[f] = a.dJ[o];
    }
    for (int f = tid; f < a.ns; f += nt) {
        long long o = (long long)f * a.rows + row;
        sh[f] = a.a1[o];
        se[f] = a.fs[o];
        sp[f] = a.fp[o];
    }
    __syncthreads();
    T acc[ITEMS];
    const T *xr = X + (long long)row * len;
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        int i = c0 + tid + it * nt;
        acc[it] = a.hd && i < c1 ? a.hd[(long long)row * len + i] * xr[i] : T(0);
    }
#pragma unroll 2
    for (int f = 0; f < a.nd; f++) {
        const T h = dh[f];
        const T *src = X + (long long)dj[f] * len;
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int i = c0 + tid + it * nt;
            if (i < c1) acc[it] += h * src[i];
        }
    }
    for (int f = 0; f < a.ns; f++) {
        const uint32_t e = se[f];
        const T h = sh[f];
        const T *src = X + (long long)(e & 0x3fffffffu) * len;
        const T *jr = a.jc + (long long)sp[f] * len;
#pragma unroll
        for (int it = 0; it < ITEMS; it++) {
            int i = c0 + tid + it * nt;
            if (i < c1) acc[it] += flip(h + jr[i], e >> 31) * src[i];
        }
    }
    T *yr = Y + (long long)row * len;
#pragma unroll
    for (int it = 0; it < ITEMS; it++) {
        int i = c0 + tid + it * nt;
        if (i < c1) yr[i] = acc[it];
    }
}

static size_t stream_smem(int nd, int ns, size_t w) {
    return (size_t)nd * (w + 4) + (size_t)ns * (w + 8) + 16;
}

// Column segments per row: the fewest that keep a thread at <= 16 items
// with up to 256 threads per CTA, <= 8 with more (register budget).
static int stream_segment(int len, int nt) {
    int cap = nt > 256 ? 8 : 16;
    int nseg = (len + nt * cap - 1) / (nt * cap);
    int seg = (len + nseg - 1) / nseg;
    return (seg + 31) / 32 * 32;
}

template <typename T>
static jci_status launch_stream(const StreamArgs<T> &a, int nt, const T *x, T *y,
                                cudaStream_t st) {
    const int seg = stream_segment(a.len, nt);
    const int items = (seg + nt - 1) / nt;
    dim3 grid(a.rows, (a.len + seg - 1) / seg);
    size_t smem = stream_smem(a.nd, a.ns, sizeof(T));
#define JCI_STREAM(IT)                                                                 \
    if (items <= IT) {                                                                 \
        JCI_CUDA(smem_optin(k_sigma_stream<T, IT>));                                   \
        k_sigma_stream<T, IT><<<grid, nt, smem, st>>>(a, seg, x, y);                   \
        return JCI_OK;                                                                 \
    }
    JCI_STREAM(1)
    JCI_STREAM(2)
    JCI_STREAM(4)
    JCI_STREAM(8)
    JCI_STREAM(16)
#undef JCI_STREAM
    return JCI_ERR_ARG;
}

static bool stream_ok(int len, int nt) {
    return (nt == 128 || nt == 256 || nt == 512 || nt == 1024) &&
           !(nt > 32 * ((len + 31) / 32) && nt > 128);
}

static size_t rows_smem(int nb, int npair, int da, int RB, size_t w) {
    return (size_t)RB * nb * w + (size_t)RB * npair * w + (size_t)RB * da * (w + 4) + 16;
}

// Dynamic shared memory of k_sigma_mixed / k_sigma_wave (nb B buffers; with
// the compact panel, cp_rows = mrows chunk masks and bases); it also covers
// k_sigma_mixed_blk's unpadded layout with two buffers.
static size_t mix_smem(int K, int TM, size_t w, int nb = 2, int cp_rows = 0) {
    const int K4 = mix_k4(K, (int)w);
    return (size_t)K4 * mix_as(TM, (int)w) * w + (size_t)nb * K4 * mix_bs((int)w) * w +
           (size_t)((K + 1) & ~1) * 4 + (size_t)cp_rows * 12 + 16;
}

static size_t fci_smem(int nb, int npair, int R, size_t w) {
    return (size_t)(1 + R) * nb * w + (size_t)R * npair * w + (size_t)npair * w +
           (size_t)R * (w + 8) + 64;
}

template <typename T, int ITEMS>
static jci_status set_smem_attr(size_t) {
    JCI_CUDA(smem_optin(k_sigma_fci<T, ITEMS>));
    return JCI_OK;
}

jci_status fci_prepare(jci_space *s) {
    DeviceState *d = s->dev;
    if (!d->single_group) return JCI_OK;
    const SpinSpace &A = s->sp[0], &B = s->sp[1];
    if (A.nstr >= (1 << 30) || B.nstr >= (1 << 30) || d->npair > 65535) return JCI_OK;
    if (B.nstr > 32 * 512) return JCI_OK;  // register-resident row limit
    cudaStream_t st = d->stream;
    FciTables *f = d->fci;
    if (!f) {
        f = new FciTables();
        d->fci = f;
        f->na = A.nstr; f->nb = B.nstr;
        f->sa = A.max_sing; f->sb = B.max_sing;
        f->da = A.max_doub; f->db = B.max_doub;
        f->npair = d->npair;
        f->nelb = B.nelec;
        for (int sp = 0; sp < 2; sp++) {
            const SpinSpace &X = s->sp[sp];
            size_t n = (size_t)X.nstr;
            size_t ns = (size_t)X.max_sing * n + 1, nd = (size_t)X.max_doub * n + 1;
            size_t npn = (size_t)d->npair * n;
            JCI_CUDA(cudaMalloc(&f->dblJ[sp], nd * sizeof(int)));
            JCI_CUDA(cudaMalloc(&f->d[sp].a1T, ns * sizeof(double)));
            JCI_CUDA(cudaMalloc(&f->d[sp].joccT, npn * sizeof(double)));
            JCI_CUDA(cudaMalloc(&f->d[sp].dblH, nd * sizeof(double)));
            JCI_CUDA(cudaMalloc(&f->f[sp].a1T, ns * sizeof(float)));
            JCI_CUDA(cudaMalloc(&f->f[sp].joccT, npn * sizeof(float)));
            JCI_CUDA(cudaMalloc(&f->f[sp].dblH, nd * sizeof(float)));
        }
        int dev = d->device, optin = 0;
        JCI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        f->smem_max = (size_t)optin;
        // the kernel needs at least the own row plus one staged row
        if (fci_smem(f->nb, f->npair, 1, sizeof(double)) > f->smem_max) f->smem_max = 0;
        // beta singles of every string sorted by target, for k_sigma_mixed2
        if (B.nstr < 65536 && d->npair < 32768 && B.max_sing < 256) {
            std::vector<uint32_t> so((size_t)B.nstr * B.max_sing);
            for (int i = 0; i < B.nstr; i++) {
                uint32_t *row = &so[(size_t)i * B.max_sing];
                for (int k = 0; k < B.max_sing; k++) {
                    const Exc &x = B.sing[B.soff[i] + k];
                    row[k] = (uint32_t)x.target | ((uint32_t)pair_index(x.io0, x.fo0) << 16) |
                             (x.sign < 0 ? 0x80000000u : 0u);
                }
                std::sort(row, row + B.max_sing,
                          [](uint32_t u, uint32_t w) { return (u & 0xffffu) < (w & 0xffffu); });
            }
            JCI_CUDA(cudaMalloc(&f->sortB, so.size() * sizeof(uint32_t)));
            JCI_CUDA(cudaMemcpy(f->sortB, so.data(), so.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice));
        }
        JCI_CUDA(cudaMalloc(&f->tc_status, sizeof(int)));
        JCI_CUDA(cudaMemset(f->tc_status, 0, sizeof(int)));
    }
    for (int sp = 0; sp < 2; sp++) {
        const SpinTables &t = d->t[sp];
        const SpinSpace &X = s->sp[sp];
        k_fci_tables<<<(X.nstr + 127) / 128, 128, 0, st>>>(
            X.nstr, X.nelec, X.max_sing, X.max_doub, d->npair, t.istr, t.doub, t.a1, d->m2,
            f->d[sp].a1T, f->f[sp].a1T, f->d[sp].joccT, f->f[sp].joccT, f->dblJ[sp],
            f->d[sp].dblH, f->f[sp].dblH);
        // the group coefficient blocks and the pair matrices follow the
        // current integrals
        if (f->grp[sp].uidx) {
            jci_status r = group_fill(&f->grp[sp], f->d[sp].dblH, f->f[sp].dblH, st);
            if (r) return r;
        }
        if (f->prs[sp].jrow) {
            jci_status r = pair_fill(s, &f->prs[sp], st);
            if (r) return r;
        }
        if (sp == 1 && f->hst.srow) {
            jci_status r = hs_fill(&f->hst, f->d[1].a1T, f->f[1].a1T, st);
            if (r) return r;
        }
    }
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

template <typename T>
static jci_status launch_one(const FciArgs<T> &a, int nt, size_t smem, int na, const T *v, T *o,
                             cudaStream_t st) {
    int items = (a.nb + nt - 1) / nt;
    jci_status r = JCI_OK;
    dim3 grid(na);
#define JCI_LAUNCH(IT)                                                          \
    do {                                                                        \
        if ((r = set_smem_attr<T, IT>(smem)) != JCI_OK) return r;              \
        k_sigma_fci<T, IT><<<grid, nt, smem, st>>>(a, v, o);                    \
    } while (0)
    if (items <= 2) JCI_LAUNCH(2);
    else if (items <= 4) JCI_LAUNCH(4);
    else if (items <= 8) JCI_LAUNCH(8);
    else if (items <= 16) JCI_LAUNCH(16);
    else JCI_LAUNCH(32);
#undef JCI_LAUNCH
    return JCI_OK;
}

template <typename T, int IT, int RB>
static jci_status launch_rows_t(const FciArgs<T> &a, int nt, const T *v, T *o,
                                cudaStream_t st) {
    size_t smem = rows_smem(a.nb, a.npair, a.da, RB, sizeof(T));
    JCI_CUDA(smem_optin(k_sigma_rows<T, IT, RB>));
    k_sigma_rows<T, IT, RB><<<(a.na + RB - 1) / RB, nt, smem, st>>>(a, v, o);
    return JCI_OK;
}

// Row kernel of the dense-product plan with nt threads and RB rows per CTA.
template <typename T>
static jci_status launch_rows(const FciArgs<T> &a, int nt, int RB, const T *v, T *o,
                              cudaStream_t st) {
    int items = (a.nb + nt - 1) / nt;
    int IT = items <= 2 ? 2 : items <= 4 ? 4 : items <= 8 ? 8 : items <= 16 ? 16 : 32;
    if (items > 32 || IT * RB > 32) return JCI_ERR_ARG;
    if (nt > (IT * RB <= 4 ? 1024 : 512)) return JCI_ERR_ARG;
#define JCI_ROWS(I, B) \
    if (IT == I && RB == B) return launch_rows_t<T, I, B>(a, nt, v, o, st)
    JCI_ROWS(2, 1); JCI_ROWS(2, 2); JCI_ROWS(2, 4);
    JCI_ROWS(4, 1); JCI_ROWS(4, 2); JCI_ROWS(4, 4);
    JCI_ROWS(8, 1); JCI_ROWS(8, 2); JCI_ROWS(8, 4);
    JCI_ROWS(16, 1); JCI_ROWS(16, 2);
    JCI_ROWS(32, 1);
#undef JCI_ROWS
    return JCI_ERR_ARG;
}

static bool rows_ok(int nb, int nt, int RB) {
    int items = (nb + nt - 1) / nt;
    int IT = items <= 2 ? 2 : items <= 4 ? 4 : items <= 8 ? 8 : items <= 16 ? 16 : 32;
    if (items > 32 || IT * RB > 32) return false;
    if (RB != 1 && RB != 2 && RB != 4) return false;
    if (nt != 128 && nt != 256 && nt != 512 && nt != 1024) return false;
    return nt <= (IT * RB <= 4 ? 1024 : 512);
}

template <typename T>
using MixKernel = void (*)(MixArgs<T>, const T *, T *, T *);

template <typename T>
static MixKernel<T> mixed_kernel(int TM) {
    switch (TM) {
        case 1: return k_sigma_mixed<T, 1>;
        case 2: return k_sigma_mixed<T, 2>;
        case 3: return k_sigma_mixed<T, 3>;
        case 4: return k_sigma_mixed<T, 4>;
        case 5: return k_sigma_mixed<T, 5>;
        case 6: return k_sigma_mixed<T, 6>;
        case 7: return k_sigma_mixed<T, 7>;
        case 8: return k_sigma_mixed<T, 8>;
        case 9: return k_sigma_mixed<T, 9>;
        default: return nullptr;
    }
}

template <typename T>
static MixKernel<T> mixed_kernel1(int TM) {
    switch (TM) {
        case 1: return k_sigma_mixed<T, 1, 1>;
        case 2: return k_sigma_mixed<T, 2, 1>;
        case 3: return k_sigma_mixed<T, 3, 1>;
        case 4: return k_sigma_mixed<T, 4, 1>;
        case 5: return k_sigma_mixed<T, 5, 1>;
        case 6: return k_sigma_mixed<T, 6, 1>;
        case 7: return k_sigma_mixed<T, 7, 1>;
        case 8: return k_sigma_mixed<T, 8, 1>;
        case 9: return k_sigma_mixed<T, 9, 1>;
        default: return nullptr;
    }
}

static bool mixed_possible(const FciTables *f, size_t w) {
    int mrows = f->npair + 1, TM = (mrows + 15) / 16;
    return TM <= 9 && f->sa >= 1 && mix_smem(f->sa, TM, w) <= f->smem_max;
}

static jci_status ab_tables(jci_space *s, int tx, cudaStream_t st, AbTables **out);

template <typename T, int TM>
static jci_status launch_mixed_blk_t(jci_space *s, const MixBArgs<T> &ab, const T *v, T *o,
                                     cudaStream_t st, int per_sm) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    auto kern = k_sigma_mixed_blk<T, TM>;
    size_t smem = mix_smem(ab.m.sa, TM, sizeof(T));
    JCI_CUDA(smem_optin(kern));
    int occ = 0, nsm = 0;
    JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMixThreads, smem));
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device));
    occ = std::max(occ, 1);
    if (!f->mixk_grid[prec]) {  // scratch blocks for the largest resident grid, once
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        JCI_CUDA(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
        const int g = std::max(1, std::min(ab.m.na, nsm * occ));
        JCI_CUDA(cudaMalloc(&f->tbufk[prec], (size_t)g * ab.m.mrows * kMixBlock * sizeof(T)));
        f->mixk_grid[prec] = g;
    }
    int grid = f->mixk_grid[prec];
    if (per_sm > 0 && per_sm < occ) grid = std::max(1, std::min(grid, nsm * per_sm));
    kern<<<grid, kMixThreads, smem, st>>>(ab, v, o, (T *)f->tbufk[prec]);
    return JCI_OK;
}

// The product through the column-blocked panel (k_sigma_mixed_blk) with
// per_sm CTAs per SM (0 = as many as fit).
template <typename T>
static jci_status launch_mixed_blk(jci_space *s, const MixArgs<T> &m, const T *v, T *o,
                                   cudaStream_t st, int per_sm) {
    AbTables *t = nullptr;
    jci_status r = ab_tables(s, kMixBlock / 4, st, &t);
    if (r) return r;
    MixBArgs<T> ab;
    ab.m = m;
    ab.offs = t->offs;
    ab.off = t->off;
    ab.base = t->base;
    ab.ent = t->ent;
    switch ((m.mrows + 15) / 16) {
        case 1: return launch_mixed_blk_t<T, 1>(s, ab, v, o, st, per_sm);
        case 2: return launch_mixed_blk_t<T, 2>(s, ab, v, o, st, per_sm);
        case 3: return launch_mixed_blk_t<T, 3>(s, ab, v, o, st, per_sm);
        case 4: return launch_mixed_blk_t<T, 4>(s, ab, v, o, st, per_sm);
        case 5: return launch_mixed_blk_t<T, 5>(s, ab, v, o, st, per_sm);
        case 6: return launch_mixed_blk_t<T, 6>(s, ab, v, o, st, per_sm);
        case 7: return launch_mixed_blk_t<T, 7>(s, ab, v, o, st, per_sm);
        case 8: return launch_mixed_blk_t<T, 8>(s, ab, v, o, st, per_sm);
        case 9: return launch_mixed_blk_t<T, 9>(s, ab, v, o, st, per_sm);
        default: return JCI_ERR_SPACE;
    }
}

// Test hook: start the queue past the GEMM items of the first kWaveLag rows,
// so that nothing ever completes them and the gathers of those rows wait
// until their bounded waits expire.
__global__ void k_wave_arm(WaveCtl *ctl, int first) { ctl->next = first; }

template <typename T>
using WaveKernel = void (*)(MixArgs<T>, const T *, T *, T *, WaveCtl *, int, int, int *);

template <typename T, int NB>
static WaveKernel<T> wave_kernel(int TM) {
    switch (TM) {
        case 1: return k_sigma_wave<T, 1, NB>;
        case 2: return k_sigma_wave<T, 2, NB>;
        case 3: return k_sigma_wave<T, 3, NB>;
        case 4: return k_sigma_wave<T, 4, NB>;
        case 5: return k_sigma_wave<T, 5, NB>;
        case 6: return k_sigma_wave<T, 6, NB>;
        case 7: return k_sigma_wave<T, 7, NB>;
        case 8: return k_sigma_wave<T, 8, NB>;
        case 9: return k_sigma_wave<T, 9, NB>;
        default: return nullptr;
    }
}

// The product through row panels shared by all CTAs (k_sigma_wave) with
// per_sm CTAs per SM (0 = as many as fit).  The kWaveBufs panels and the
// queue counters are allocated on first use; the counters are cleared on
// the stream before every launch.
template <typename T>
static jci_status launch_wave(jci_space *s, const MixArgs<T> &m, const T *v, T *o,
                              cudaStream_t st, int per_sm) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    const int TM = (m.mrows + 15) / 16;
    WaveKernel<T> kern = wave_kernel<T, 2>(TM), kern1 = wave_kernel<T, 1>(TM);
    if (!kern || !kern1) return JCI_ERR_SPACE;
    size_t smem = mix_smem(m.sa, TM, sizeof(T)), smem1 = mix_smem(m.sa, TM, sizeof(T), 1);
    if (smem + 64 > f->smem_max) return JCI_ERR_SPACE;  // 16 bytes of static shared memory
    JCI_CUDA(smem_optin(kern));
    JCI_CUDA(smem_optin(kern1));
    int occ = 0, occ1 = 0, nsm = 0;
    JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMixThreads, smem));
    JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, kern1, kMixThreads, smem1));
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device));
    if (occ < 2 && occ1 > occ) {  // one B buffer when that lets a second CTA share each SM
        kern = kern1;
        smem = smem1;
        occ = occ1;
    }
    if (occ < 1) return JCI_ERR_SPACE;
    const int nchunk = m.nbp / kMixCols;
    const int ngi = (nchunk + kWaveChunks - 1) / kWaveChunks;
    const int nhi = (m.nb + kMixThreads - 1) / kMixThreads;
    int grid = nsm * (per_sm > 0 && per_sm < occ ? per_sm : occ);
    if ((long long)m.na * (ngi + nhi) + grid >= (1ll << 31)) return JCI_ERR_SPACE;
    if (!f->wbuf[prec]) {
        JCI_CUDA(cudaMalloc(&f->wbuf[prec], (size_t)kWaveBufs * m.mrows * m.nbp * sizeof(T)));
        JCI_CUDA(cudaMalloc(&f->wctl[prec], sizeof(WaveCtl)));
    }
    JCI_CUDA(cudaMemsetAsync(f->wctl[prec], 0, sizeof(WaveCtl), st));
    if (f->wave_expire) {
        f->wave_expire = 0;
        k_wave_arm<<<1, 1, 0, st>>>((WaveCtl *)f->wctl[prec], std::min(kWaveLag, m.na) * ngi);
    }
    kern<<<grid, kMixThreads, smem, st>>>(m, v, o, (T *)f->wbuf[prec], (WaveCtl *)f->wctl[prec],
                                          ngi, nhi, f->tc_status);
    return JCI_OK;
}

// Tables of the compact product panel (integral independent), built on the
// host on first use, not while a stream is being captured.  A panel entry
// (row m, column J) is kept iff the gather reads it: the one-body row at
// every column, the Coulomb row (mm) at the strings that hold m, and the
// single pair row at every single's target.  At FCI(16,16) that is 73 of
// the 137 rows per column.  Positions run row after row, columns ascending.
static jci_status compact_tables(jci_space *s, cudaStream_t st) {
    FciTables *f = s->dev->fci;
    if (f->cp_state > 0) return JCI_OK;
    if (f->cp_state < 0) return JCI_ERR_SPACE;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    JCI_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
    const SpinSpace &B = s->sp[1];
    const int nb = B.nstr, ne = B.nelec, sb = f->sb, mrows = f->npair + 1;
    const int nchunk = (nb + kMixCols - 1) / kMixCols;
    f->cp_state = -1;
    for (int i = 0; i < nb; i++)
        if (B.soff[i + 1] - B.soff[i] != sb) return JCI_ERR_SPACE;
    // the gather's reads of string Ib, in its summation order: (row, column, phase)
    const int gent = 1 + ne + sb;
    std::vector<int> grow((size_t)gent * nb), gcol((size_t)gent * nb), gneg((size_t)gent * nb);
    for (int i = 0; i < nb; i++) {
        int e = 0;
        auto put = [&](int row, int col, int neg) {
            grow[(size_t)e * nb + i] = row;
            gcol[(size_t)e * nb + i] = col;
            gneg[(size_t)e * nb + i] = neg;
            e++;
        };
        put(f->npair, i, 0);
        // Coulomb rows in ascending orbital order (the order of the occupation bits)
        for (int k = 0; k < ne; k++) {
            const int o = B.istr[(size_t)i * ne + k];
            if (o > 64) return JCI_ERR_SPACE;
            put(pair_index(o, o), i, 0);
        }
        for (int k = 0; k < sb; k++) {
            const Exc &x = B.sing[B.soff[i] + k];
            put(pair_index(x.io0, x.fo0), x.target, x.sign < 0);
        }
    }
    std::vector<uint64_t> mask((size_t)nchunk * mrows, 0);
    for (size_t q = 0; q < grow.size(); q++)
        mask[(size_t)(gcol[q] >> 6) * mrows + grow[q]] |= 1ull << (gcol[q] & 63);
    // positions: row after row, chunk after chunk within a row
    std::vector<int> base((size_t)nchunk * mrows);
    long long pos = 0;
    for (int m = 0; m < mrows; m++)
        for (int c = 0; c < nchunk; c++) {
            base[(size_t)c * mrows + m] = (int)pos;
            pos += __builtin_popcountll(mask[(size_t)c * mrows + m]);
        }
    if (pos >= (1ll << 31)) return JCI_ERR_SPACE;
    std::vector<int> gidx((size_t)gent * nb);
    for (size_t q = 0; q < grow.size(); q++) {
        const size_t k = (size_t)(gcol[q] >> 6) * mrows + grow[q];
        const int p = base[k] + __builtin_popcountll(mask[k] & ((1ull << (gcol[q] & 63)) - 1));
        gidx[q] = p | (gneg[q] ? (int)0x80000000u : 0);
    }
    JCI_CUDA(cudaMalloc(&f->cp_mask, mask.size() * sizeof(uint64_t)));
    JCI_CUDA(cudaMalloc(&f->cp_base, base.size() * sizeof(int)));
    JCI_CUDA(cudaMalloc(&f->cp_gidx, gidx.size() * sizeof(int)));
    JCI_CUDA(cudaMemcpy(f->cp_mask, mask.data(), mask.size() * sizeof(uint64_t),
                        cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(f->cp_base, base.data(), base.size() * sizeof(int),
                        cudaMemcpyHostToDevice));
    JCI_CUDA(cudaMemcpy(f->cp_gidx, gidx.data(), gidx.size() * sizeof(int),
                        cudaMemcpyHostToDevice));
    f->cp_len = pos;
    f->cp_ent = gent;
    f->cp_state = 1;
    return JCI_OK;
}

// Second kernel of the dense-product path.  The per-CTA scratch panels are
// allocated on first use for the largest resident grid; `per_sm` picks the
// CTAs per SM actually launched (0 = as many as fit), which trades latency
// hiding against keeping the panels L2-resident.  per_sm >= 16 selects the
// column-blocked panel (k_sigma_mixed_blk) with per_sm - 16 CTAs per SM,
// per_sm >= 32 the row-shared panels (k_sigma_wave) with per_sm - 32, and
// per_sm >= 64 the compact panel (compact_tables) with per_sm - 64.
template <typename T>
static jci_status launch_mixed(jci_space *s, const FciArgs<T> &fa, const T *v, T *o,
                               cudaStream_t st, int per_sm) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    MixArgs<T> m;
    m.na = fa.na; m.nb = fa.nb; m.nbp = (fa.nb + kMixCols - 1) / kMixCols * kMixCols;
    m.sa = fa.sa; m.sb = fa.sb; m.npair = fa.npair; m.mrows = fa.npair + 1;
    m.fsA = fa.fsA; m.fsB = fa.fsB; m.fpA = fa.fpA; m.fpB = fa.fpB;
    m.a1A = fa.a1A; m.m2 = fa.m2; m.occB = d->t[1].occ;
    m.skip = fa.skip;
    int cp_rows = 0;
    if (per_sm >= 64) {
        jci_status r = compact_tables(s, st);
        if (r) return r;
        m.cmask = f->cp_mask;
        m.cbase = f->cp_base;
        m.gidx = f->cp_gidx;
        m.gent = f->cp_ent;
        m.plen = f->cp_len;
        cp_rows = m.mrows;
        per_sm -= 64;
        if (per_sm >= 16) return JCI_ERR_ARG;  // whole-row panels only
    }
    if (per_sm >= 32) return launch_wave<T>(s, m, v, o, st, per_sm - 32);
    if (per_sm >= 16) return launch_mixed_blk<T>(s, m, v, o, st, per_sm - 16);
    int TM = (m.mrows + 15) / 16;
    MixKernel<T> kern = mixed_kernel<T>(TM), kern1 = mixed_kernel1<T>(TM);
    if (!kern || !kern1) return JCI_ERR_SPACE;
    size_t smem = mix_smem(m.sa, TM, sizeof(T), 2, cp_rows),
           smem1 = mix_smem(m.sa, TM, sizeof(T), 1, cp_rows);
    if (smem1 > f->smem_max) return JCI_ERR_SPACE;
    JCI_CUDA(smem_optin(kern));
    JCI_CUDA(smem_optin(kern1));
    {
        // one B buffer when that lets a second CTA share each SM
        int occ2 = 0, occ1 = 0;
        JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, kern, kMixThreads, smem));
        JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, kern1, kMixThreads, smem1));
        if (occ2 < 2 && occ1 > occ2) {
            kern = kern1;
            smem = smem1;
        }
    }
    if (!f->mix_grid[prec]) {
        int occ = 0, nsm = 0;
        JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMixThreads, smem));
        JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device));
        int grid = std::max(1, std::min(m.na, nsm * std::max(occ, 1)));
        size_t bytes = (size_t)grid * m.mrows * m.nbp * sizeof(T);
        JCI_CUDA(cudaMalloc(&f->tbuf[prec], bytes));
        f->mix_grid[prec] = grid;
        f->mix_occ[prec] = std::max(occ, 1);
        f->nsm = nsm;
    }
    int grid = f->mix_grid[prec];
    if (per_sm > 0 && per_sm < f->mix_occ[prec])
        grid = std::max(1, std::min(grid, f->nsm * per_sm));
    if (cp_rows) {  // no more CTAs than fit with the masks' shared memory
        int occ = 0;
        JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMixThreads, smem));
        grid = std::max(1, std::min(grid, f->nsm * std::max(occ, 1)));
    }
    kern<<<grid, kMixThreads, smem, st>>>(m, v, o, (T *)f->tbuf[prec]);
    return JCI_OK;
}

template <typename T>
using Mix2Kernel = void (*)(Mix2Args<T>, const T *, T *);

template <typename T>
static Mix2Kernel<T> mixed2_kernel(int TM) {
    switch (TM) {
        case 1: return k_sigma_mixed2<T, 1>;
        case 2: return k_sigma_mixed2<T, 2>;
        case 3: return k_sigma_mixed2<T, 3>;
        case 4: return k_sigma_mixed2<T, 4>;
        case 5: return k_sigma_mixed2<T, 5>;
        case 6: return k_sigma_mixed2<T, 6>;
        case 7: return k_sigma_mixed2<T, 7>;
        case 8: return k_sigma_mixed2<T, 8>;
        case 9: return k_sigma_mixed2<T, 9>;
        default: return nullptr;
    }
}

static bool mixed2_possible(const FciTables *f, size_t w) {
    int mrows = f->npair + 1, TM = (mrows + 15) / 16;
    return f->sortB && TM <= 9 && f->sa >= 1 &&
           mix2_smem(f->sa, TM, mrows, f->nb, w) <= f->smem_max;
}

// Panel-free product kernel with per_sm CTAs per SM (0 = as many as fit).
template <typename T>
static jci_status launch_mixed2(jci_space *s, const FciArgs<T> &fa, const T *v, T *o,
                                cudaStream_t st, int per_sm) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    Mix2Args<T> m;
    m.na = fa.na; m.nb = fa.nb; m.nbp = (fa.nb + kMixCols - 1) / kMixCols * kMixCols;
    m.sa = fa.sa; m.sb = fa.sb; m.npair = fa.npair; m.mrows = fa.npair + 1;
    m.fsA = fa.fsA; m.fpA = fa.fpA; m.sortB = f->sortB;
    m.a1A = fa.a1A; m.m2 = fa.m2; m.occB = d->t[1].occ;
    m.skip = fa.skip;
    int TM = (m.mrows + 15) / 16;
    Mix2Kernel<T> kern = mixed2_kernel<T>(TM);
    if (!kern || !f->sortB) return JCI_ERR_SPACE;
    size_t smem = mix2_smem(m.sa, TM, m.mrows, m.nb, sizeof(T));
    JCI_CUDA(smem_optin(kern));
    int occ = 0, nsm = 0;
    JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMixThreads, smem));
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device));
    occ = std::max(occ, 1);
    if (per_sm > 0) occ = std::min(occ, per_sm);
    int grid = std::max(1, std::min(m.na, nsm * occ));
    kern<<<grid, kMixThreads, smem, st>>>(m, v, o);
    return JCI_OK;
}

// Product engines of the fused plans (4, 5, 7): tx = 8 or 16 column threads
// of jci_fci_ab.cu, or 32 / 64 = the FP32 tcgen05 engine (jci_fci_tc.cu) with
// chunks of that many columns.
static bool is_tc_engine(int tx) { return tx == 32 || tx == 64; }
// Column threads whose entry lists an engine reads (chunks of 4 tx columns).
static int ab_table_tx(int tx) { return is_tc_engine(tx) ? tx / 4 : tx; }

static bool ab_plan_possible(const FciTables *f, int tx, size_t w) {
    const AbShape sh{f->nb, f->sa, f->sb, f->nelb, f->npair};
    if (is_tc_engine(tx)) return w == sizeof(float) && tc_possible(sh, tx, f->smem_max);
    return ab_possible(sh, tx, w, f->smem_max);
}

// Entry lists of the fused product with tx column threads, built on first use
// (not while a stream is being captured).
static jci_status ab_tables(jci_space *s, int tx, cudaStream_t st, AbTables **out) {
    if (tx != 8 && tx != 16 && tx != kMixBlock / 4) return JCI_ERR_ARG;
    FciTables *f = s->dev->fci;
    AbTables &t = tx == kMixBlock / 4 ? f->abk : f->ab[tx == 16 ? 1 : 0];
    if (!t.ent) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        JCI_CUDA(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
        jci_status r = ab_tables_build(s, f->npair, tx, &t);
        if (r) return r;
    }
    *out = &t;
    return JCI_OK;
}

// Fused product kernel (jci_fci_ab.cu) with tx column threads.
template <typename T>
static jci_status launch_ab(jci_space *s, const FciArgs<T> &fa, const T *v, T *o,
                            cudaStream_t st, int tx) {
    AbTables *t = nullptr;
    const bool tc = is_tc_engine(tx);
    jci_status r = ab_tables(s, ab_table_tx(tx), st, &t);
    if (r) return r;
    AbArgs<T> m;
    m.na = fa.na; m.nb = fa.nb; m.sa = fa.sa; m.npair = fa.npair; m.mrows = fa.npair + 1;
    m.nchunk = t->nchunk;
    m.offs = t->offs;
    m.maxent = t->maxent;
    m.vec = ((size_t)fa.nb * sizeof(T) % 16 == 0 && reinterpret_cast<uintptr_t>(v) % 16 == 0) ? 1 : 0;
    m.fsA = fa.fsA; m.fpA = fa.fpA; m.a1A = fa.a1A; m.m2 = fa.m2;
    m.off = t->off; m.base = t->base; m.ent = t->ent;
    m.skip = fa.skip;
    if constexpr (sizeof(T) == sizeof(float)) {
        if (tc) {
            return tc_launch(m, tx, s->dev->device, v, o, s->dev->fci->tc_status, st);
        }
    }
    if (tc) return JCI_ERR_ARG;
    return ab_launch<T>(m, tx, s->dev->device, v, o, st);
}

// Group tables of both spins, built and filled on first use (not while a
// stream is being captured).
static jci_status group_tables(jci_space *s, cudaStream_t st) {
    FciTables *f = s->dev->fci;
    for (int sp = 0; sp < 2; sp++) {
        if (f->grp[sp].uidx) continue;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        JCI_CUDA(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
        jci_status r = group_tables_build(s, sp, &f->grp[sp]);
        if (!r) r = group_fill(&f->grp[sp], f->d[sp].dblH, f->f[sp].dblH, st);
        if (r) {
            group_tables_free(&f->grp[0]);
            group_tables_free(&f->grp[1]);
            return r;
        }
    }
    return JCI_OK;
}

static bool group_possible(const FciTables *f) { return f->da >= 1 && f->db >= 1; }

// Hole-string tables of both spins (jci_fci_pairs.cu), built and filled on
// first use (not while a stream is being captured); JCI_ERR_SPACE, and
// remembered, for spaces they do not cover.
static jci_status pair_tables(jci_space *s, cudaStream_t st) {
    FciTables *f = s->dev->fci;
    if (f->prs_state > 0) return JCI_OK;
    if (f->prs_state < 0) return JCI_ERR_SPACE;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    JCI_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
    jci_status r = JCI_OK;
    for (int sp = 0; sp < 2 && !r; sp++) {
        r = pair_tables_build(s, sp, &f->prs[sp]);
        if (!r) r = pair_fill(s, &f->prs[sp], st);
        if (!r && pair_smem_bytes(f->prs[sp], 0) > f->smem_max) r = JCI_ERR_SPACE;
    }
    if (r) {
        pair_tables_free(&f->prs[0]);
        pair_tables_free(&f->prs[1]);
        f->prs_state = r == JCI_ERR_SPACE ? -1 : 0;
        return r;
    }
    f->prs_state = 1;
    return JCI_OK;
}

// Beta-singles tables through hole strings (jci_fci_pairs.cu), built and
// filled on first use (not while a stream is being captured); JCI_ERR_SPACE,
// and remembered, for spaces they do not cover.
static jci_status hs_tables(jci_space *s, cudaStream_t st) {
    FciTables *f = s->dev->fci;
    if (f->hs_state > 0) return JCI_OK;
    if (f->hs_state < 0) return JCI_ERR_SPACE;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    JCI_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
    jci_status r = hs_tables_build(s, 1, &f->hst);
    if (!r) r = hs_fill(&f->hst, f->d[1].a1T, f->f[1].a1T, st);
    if (!r && hs_smem_bytes(f->npair, sizeof(double)) > f->smem_max) r = JCI_ERR_SPACE;
    if (r) {
        hs_tables_free(&f->hst);
        f->hs_state = r == JCI_ERR_SPACE ? -1 : 0;
        return r;
    }
    f->hs_state = 1;
    return JCI_OK;
}

// The beta singles of plans 6 and 7 with threads = 0: through the hole
// strings of the beta strings, on C^T (rows Ib) into tau (overwritten).
template <typename T>
static jci_status launch_hs(jci_space *s, const StreamArgs<T> &be, const T *ct, T *tau,
                            cudaStream_t st) {
    FciTables *f = s->dev->fci;
    jci_status r = hs_tables(s, st);
    if (r) return r;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    const size_t need =
        (size_t)f->hst.nk * f->hst.nf * hs_block_cols(f->hst, f->na, sizeof(T)) * sizeof(T);
    if (f->hbytes[prec] < need) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        JCI_CUDA(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
        JCI_CUDA(cudaFree(f->hbuf[prec]));
        f->hbuf[prec] = nullptr;
        f->hbytes[prec] = 0;
        JCI_CUDA(cudaMalloc(&f->hbuf[prec], need));
        f->hbytes[prec] = need;
    }
    return hs_launch<T>(f->hst, f->na, f->npair, be.jc, ct, tau, be.skip, (T *)f->hbuf[prec],
                        s->dev->device, st);
}

// E block of the hole-string doubles for variant `items` (5, 6) in this
// precision, grown on demand (not while a stream is being captured).
template <typename T>
static jci_status pair_scratch(jci_space *s, int items, cudaStream_t st, T **E) {
    FciTables *f = s->dev->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    size_t need = 0;
    for (int sp = 0; sp < 2; sp++) {
        const PairTables &t = f->prs[sp];
        const int len = sp == 0 ? f->nb : f->na;
        need = std::max(need, (size_t)t.nk * t.np * pair_block_cols(t, len, items, sizeof(T)) *
                                  sizeof(T));
    }
    if (f->pbytes[prec] < need) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        JCI_CUDA(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) return JCI_ERR_STATE;
        JCI_CUDA(cudaFree(f->pbuf[prec]));
        f->pbuf[prec] = nullptr;
        f->pbytes[prec] = 0;
        JCI_CUDA(cudaMalloc(&f->pbuf[prec], need));
        f->pbytes[prec] = need;
    }
    *E = (T *)f->pbuf[prec];
    return JCI_OK;
}

// Doubles of spin sp: rows x len matrix x -> y (add: y += ...), with the
// diagonal hd when given; items = the variant: 1-4 the string-group kernel
// (group_launch), 5-7 the hole-string products (pair_launch: widest column
// block under 1 GiB of E, 64-column blocks, widest under 4 GiB).
template <typename T>
static jci_status launch_group(jci_space *s, int sp, const T *hd, int add, const int *skip,
                               int items, const T *x, T *y, cudaStream_t st) {
    FciTables *f = s->dev->fci;
    if (items >= 5) {
        jci_status r = pair_tables(s, st);
        T *E = nullptr;
        if (!r) r = pair_scratch<T>(s, items, st, &E);
        if (r) return r;
        return pair_launch<T>(f->prs[sp], sp == 0 ? f->nb : f->na, items, x, y, hd, add, skip, E,
                              s->dev->device, st);
    }
    jci_status r = group_tables(s, st);
    if (r) return r;
    const GroupTables &t = f->grp[sp];
    GroupArgs<T> g;
    g.rows = sp == 0 ? f->na : f->nb;
    g.len = sp == 0 ? f->nb : f->na;
    g.uoff = t.uoff;
    g.uidx = t.uidx;
    g.useg = t.useg;
    if constexpr (sizeof(T) == sizeof(double))
        g.coef = t.c64;
    else
        g.coef = t.c32;
    g.hd = hd;
    g.add = add;
    g.skip = skip;
    return group_launch<T>(g, items, s->dev->device, x, y, st);
}

// Scratch of the streaming plan: C^T and the beta part, N each, allocated on
// the first use of the plan (the autotuner's trial) and kept.
template <typename T>
static jci_status stream_scratch(FciTables *f, T **ct, T **tau) {
    const int prec = sizeof(T) == 8 ? 0 : 1;
    size_t n = (size_t)f->na * f->nb;
    if (!f->sbuf[prec]) JCI_CUDA(cudaMalloc(&f->sbuf[prec], 2 * n * sizeof(T)));
    *ct = (T *)f->sbuf[prec];
    *tau = *ct + n;
    return JCI_OK;
}

// alpha pass on C (rows Ia): diagonal and alpha doubles; beta pass on C^T
// (rows Ib): beta doubles and beta singles with the alpha string's Coulomb
// row jocc[pair][Ia] (hmatels_1x, action_util.c:210)
template <typename T>
static void stream_args(const FciArgs<T> &a, StreamArgs<T> &al, StreamArgs<T> &be) {
    al.rows = a.na; al.len = a.nb; al.nd = a.da; al.ns = 0;
    al.dJ = a.dJA; al.dH = a.dHA; al.fs = nullptr; al.fp = nullptr; al.a1 = nullptr;
    al.jc = nullptr; al.hd = a.hd; al.skip = a.skip;
    be.rows = a.nb; be.len = a.na; be.nd = a.db; be.ns = a.sb;
    be.dJ = a.dJB; be.dH = a.dHB; be.fs = a.fsB; be.fp = a.fpB; be.a1 = a.a1B;
    be.jc = a.jA; be.hd = nullptr; be.skip = a.skip;
}

template <typename T>
static jci_status launch_transposes(const FciTables *f, const T *v, T *ct, T *o, const T *tau,
                                    bool add, const int *skip, cudaStream_t st) {
    dim3 tb(kTile, 8), g((f->nb + kTile - 1) / kTile, (f->na + kTile - 1) / kTile);
    if (add)
        k_transpose_add<T><<<g, tb, 0, st>>>(o, f->na, f->nb, tau, skip);
    else
        k_transpose<T><<<g, tb, 0, st>>>(v, f->na, f->nb, ct, skip);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

// One full sigma of one vector with the given plan.
// mode 0: k_sigma_fci with R staged alpha rows.
// modes 1, 2, 5: k_sigma_rows (nt threads, B rows per CTA), then the product:
//   1: k_sigma_mixed with R CTAs per SM, 2: k_sigma_mixed2 with R CTAs per
//   SM, 5: the fused k_sigma_ab with R column threads (8 or 16).
// modes 3, 4: row streams on C^T (B threads) and C (nt threads), then the
//   product: 3: k_sigma_mixed (R CTAs per SM), 4: k_sigma_ab (R column
//   threads).
// modes 6, 7: the same-spin doubles by string groups on C and C^T (group
//   kernel variant B: 1 or 2 columns per thread, or 3, 4: the union split
//   over 4 warps with 2 or 1 columns per lane), the beta singles as a row
//   stream on C^T (nt threads), then the product of mode 3 (6) or of
//   mode 4 (7).
template <typename T>
static jci_status run_plan(jci_space *s, FciArgs<T> a, int mode, int nt, int R, int B,
                           const T *v, T *o, cudaStream_t st) {
    FciTables *f = s->dev->fci;
    size_t w = sizeof(T);
    jci_status r;
    if (mode == 6 || mode == 7) {
        T *ct, *tau;
        if ((r = stream_scratch<T>(f, &ct, &tau))) return r;
        StreamArgs<T> al, be;
        stream_args(a, al, be);
        be.nd = 0;  // the beta doubles come from the group kernel
        if ((r = launch_transposes<T>(f, v, ct, o, tau, false, a.skip, st))) return r;
        if ((r = nt == 0 ? launch_hs<T>(s, be, ct, tau, st) : launch_stream<T>(be, nt, ct, tau, st)))
            return r;
        if ((r = launch_group<T>(s, 1, nullptr, 1, a.skip, B, ct, tau, st))) return r;
        if ((r = launch_group<T>(s, 0, a.hd, 0, a.skip, B, v, o, st))) return r;
        if ((r = launch_transposes<T>(f, v, ct, o, tau, true, a.skip, st))) return r;
        a.do_as = 0;
        a.R = 0;
        if (mode == 7) return launch_ab<T>(s, a, v, o, st, R);
        return launch_mixed<T>(s, a, v, o, st, R);
    }
    if (mode == 3 || mode == 4) {
        // nt: threads of the alpha pass, B: threads of the beta pass
        T *ct, *tau;
        if ((r = stream_scratch<T>(f, &ct, &tau))) return r;
        StreamArgs<T> al, be;
        stream_args(a, al, be);
        if ((r = launch_transposes<T>(f, v, ct, o, tau, false, a.skip, st))) return r;
        if ((r = launch_stream<T>(be, B, ct, tau, st))) return r;
        if ((r = launch_stream<T>(al, nt, v, o, st))) return r;
        if ((r = launch_transposes<T>(f, v, ct, o, tau, true, a.skip, st))) return r;
        a.do_as = 0;
        a.R = 0;
        if (mode == 4) return launch_ab<T>(s, a, v, o, st, R);
        return launch_mixed<T>(s, a, v, o, st, R);
    }
    if (mode == 0) {
        a.do_as = 1;
        a.R = R;
        return launch_one<T>(a, nt, fci_smem(f->nb, f->npair, R, w), f->na, v, o, st);
    }
    a.do_as = 0;
    a.R = 0;
    if ((r = launch_rows<T>(a, nt, B, v, o, st))) return r;
    if (mode == 2) return launch_mixed2<T>(s, a, v, o, st, R);
    if (mode == 5) return launch_ab<T>(s, a, v, o, st, R);
    return launch_mixed<T>(s, a, v, o, st, R);
}

// Pick the plan for this space by timing the admissible candidates on
// scratch vectors (modes as in run_plan).  The row kernel, the stream passes
// and the product kernels are tuned one by one; the best configuration of
// each plan is then timed end to end.  Cached per precision.
template <typename T>
static jci_status autotune(jci_space *s, FciArgs<T> a, cudaStream_t st) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    size_t w = sizeof(T);
    long long n = (long long)f->na * f->nb;
    T *v = nullptr, *o = nullptr;
    JCI_CUDA(cudaMalloc(&v, n * w));
    JCI_CUDA(cudaMalloc(&o, n * w));
    JCI_CUDA(cudaMemsetAsync(v, 0, n * w, st));
    const int nts[] = {128, 256, 512, 1024};
    const int Rs[] = {1, 2, 4, 8, 16};
    cudaEvent_t e0, e1;
    JCI_CUDA(cudaEventCreate(&e0));
    JCI_CUDA(cudaEventCreate(&e1));
    jci_status err = JCI_OK;
    // ms per call of fn: one untimed call, then two timed -- or one, when a
    // call takes more than 50 ms (large spaces: launch noise is then far
    // below the differences between candidates, and tuning time matters)
    auto timeit = [&](auto fn) -> float {
        if (err || (err = fn())) return 1e30f;
        float ms = 0.f;
        int reps = 0;
        for (int k = 0; k < 2 && !err; k++) {
            cudaEventRecord(e0, st);
            err = fn();
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            ms += t;
            reps++;
            if (t > 50.f) break;
        }
        return err ? 1e30f : ms / reps;
    };
    auto useful = [&](int nt) {
        int items = (f->nb + nt - 1) / nt;
        return !(nt > 32 * ((f->nb + 31) / 32) && nt > 128) && items <= 32;  // idle threads
    };
    // mode 0: one kernel, R staged rows
    float best0 = 1e30f;
    int b0nt = 0, b0R = 0;
    for (int nt : nts) {
        int items = (f->nb + nt - 1) / nt;
        if (!useful(nt) || (nt == 1024 && items > 2)) continue;
        for (int R : Rs) {
            if (R > f->sa && R > 1) continue;
            if (fci_smem(f->nb, f->npair, R, w) > f->smem_max) continue;
            float ms = timeit([&] { return run_plan<T>(s, a, 0, nt, R, 1, v, o, st); });
            if (ms < best0) { best0 = ms; b0nt = nt; b0R = R; }
        }
    }
    // the product kernels (alpha singles, alpha x beta doubles), tuned on
    // their own: panel (R CTAs per SM), panel-free chunks, fused (tx)
    FciArgs<T> ar = a;
    ar.do_as = 0;
    ar.R = 0;
    float bpanel = 1e30f, bmix2 = 1e30f, bab = 1e30f;
    int Rpanel = 1, Rmix2 = 1, txab = 0;
    if (mixed_possible(f, w))
        // whole-row panel per CTA, column-blocked, row panels shared by all CTAs
        for (int R : {1, 2, 4, 16 + 1, 16 + 2, 16 + 4, 64 + 1, 64 + 2, 64 + 4}) {
            float ms = timeit([&] { return launch_mixed<T>(s, ar, v, o, st, R); });
            if (ms < bpanel) { bpanel = ms; Rpanel = R; }
        }
    if (mixed2_possible(f, w))
        for (int R : {1, 2}) {
            float ms = timeit([&] { return launch_mixed2<T>(s, ar, v, o, st, R); });
            if (ms < bmix2) { bmix2 = ms; Rmix2 = R; }
        }
    for (int tx : {8, 16, 32, 64}) {
        if (!ab_plan_possible(f, tx, w)) continue;
        float ms = timeit([&] { return launch_ab<T>(s, ar, v, o, st, tx); });
        if (ms < bab) { bab = ms; txab = tx; }
    }
    // best product behind the row kernel (modes 1, 2, 5) and behind the
    // stream passes (modes 3, 4)
    float bprod = bpanel;
    int pmode = 1, pR = Rpanel;
    if (bmix2 < bprod) { bprod = bmix2; pmode = 2; pR = Rmix2; }
    if (bab < bprod) { bprod = bab; pmode = 5; pR = txab; }
    const bool sab = bab < bpanel;
    const float bsprod = sab ? bab : bpanel;
    const int smode = sab ? 4 : 3, sR = sab ? txab : Rpanel;
    // modes 1, 2, 5: the row kernel, then the product
    float best1 = 1e30f;
    int b1nt = 0, b1B = 0, b1R = pR, b1mode = pmode;
    if (bprod < 1e30f) {
        float brow = 1e30f;
        for (int nt : nts) {
            if (!useful(nt)) continue;
            for (int B : {1, 2, 4}) {
                if (!rows_ok(f->nb, nt, B) || rows_smem(f->nb, f->npair, f->da, B, w) > f->smem_max)
                    continue;
                float ms = timeit([&] { return launch_rows<T>(ar, nt, B, v, o, st); });
                if (ms < brow) { brow = ms; b1nt = nt; b1B = B; }
            }
        }
        if (b1nt) best1 = brow + bprod;
    }
    // modes 3, 4: streaming passes on C and C^T, the transposes, the product
    float best3 = 1e30f;
    int b3a = 0, b3b = 0;
    if (bsprod < 1e30f) {
        T *ct = nullptr, *tau = nullptr;
        if (!err) err = stream_scratch<T>(f, &ct, &tau);
        StreamArgs<T> al, be;
        stream_args(a, al, be);
        float ba = 1e30f, bb = 1e30f;
        for (int nt : nts) {
            if (stream_ok(f->nb, nt) && stream_smem(al.nd, al.ns, w) <= f->smem_max) {
                float ms = timeit([&] { return launch_stream<T>(al, nt, v, o, st); });
                if (ms < ba) { ba = ms; b3a = nt; }
            }
            if (stream_ok(f->na, nt) && stream_smem(be.nd, be.ns, w) <= f->smem_max) {
                float ms = timeit([&] { return launch_stream<T>(be, nt, ct, tau, st); });
                if (ms < bb) { bb = ms; b3b = nt; }
            }
        }
        float tt = timeit([&] {
            jci_status q = launch_transposes<T>(f, v, ct, o, tau, false, nullptr, st);
            return q ? q : launch_transposes<T>(f, v, ct, o, tau, true, nullptr, st);
        });
        if (b3a && b3b) best3 = ba + bb + tt + bsprod;
    }
    // modes 6, 7: the doubles by string groups, the beta singles as a stream
    float best6 = 1e30f;
    int b6s = 0, b6i = 1;
    bool pairs = false;  // the hole-string variants (5, 6) can run
    if (bsprod < 1e30f && group_possible(f) && !err) {
        T *ct = nullptr, *tau = nullptr;
        err = stream_scratch<T>(f, &ct, &tau);
        StreamArgs<T> al, be;
        stream_args(a, al, be);
        be.nd = 0;
        float bs = 1e30f;
        bool found = false;
        for (int nt : nts) {
            if (!stream_ok(f->na, nt) || stream_smem(0, be.ns, w) > f->smem_max) continue;
            float ms = timeit([&] { return launch_stream<T>(be, nt, ct, tau, st); });
            if (ms < bs) { bs = ms; b6s = nt; found = true; }
        }
        if (hs_tables(s, st) == JCI_OK) {  // threads = 0: the beta singles through hole strings
            float ms = timeit([&] { return launch_hs<T>(s, be, ct, tau, st); });
            if (ms < bs) { bs = ms; b6s = 0; found = true; }
        }
        float gg = 1e30f;
        pairs = pair_tables(s, st) == JCI_OK;
        for (int it : {1, 2, 3, 4, 5, 6, 7}) {
            if (it >= 5 && !pairs) continue;
            float ms = timeit([&] {
                jci_status q = launch_group<T>(s, 1, nullptr, 1, nullptr, it, ct, tau, st);
                return q ? q : launch_group<T>(s, 0, a.hd, 0, nullptr, it, v, o, st);
            });
            if (ms < gg) { gg = ms; b6i = it; }
        }
        float tt = timeit([&] {
            jci_status q = launch_transposes<T>(f, v, ct, o, tau, false, nullptr, st);
            return q ? q : launch_transposes<T>(f, v, ct, o, tau, true, nullptr, st);
        });
        if (found && gg < 1e30f) best6 = bs + gg + tt + bsprod;
        err = JCI_OK;  // a space the group tables cannot hold just drops the plan
    }
    const int gmode = sab ? 7 : 6;
    // the components were timed one by one; time each plan's best
    // configuration end to end before choosing
    auto best_of = [&](auto fn) {
        float m = 1e30f;
        for (int k = 0; k < 3; k++) {
            m = std::min(m, timeit(fn));
            if (m > 50.f && m < 1e29f) break;  // as in timeit
        }
        return m;
    };
    if (b0nt) best0 = best_of([&] { return run_plan<T>(s, a, 0, b0nt, b0R, 1, v, o, st); });
    if (b1nt)
        best1 = best_of([&] { return run_plan<T>(s, a, b1mode, b1nt, b1R, b1B, v, o, st); });
    if (b3a && b3b)
        best3 = best_of([&] { return run_plan<T>(s, a, smode, b3a, sR, b3b, v, o, st); });
    if (best6 < 1e30f) {
        // every group kernel variant, end to end (their component timings
        // are close and noisy)
        best6 = 1e30f;
        for (int it : {1, 2, 3, 4, 5, 6, 7}) {
            if (it >= 5 && !pairs) continue;
            float ms = best_of([&] { return run_plan<T>(s, a, gmode, b6s, sR, it, v, o, st); });
            if (ms < best6) { best6 = ms; b6i = it; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(v);
    cudaFree(o);
    if (err) return err;
    if (!b0nt && !b1nt && !(b3a && b3b) && best6 >= 1e30f) return JCI_ERR_SPACE;
    int mode = 0;
    float best = best0;
    if (b1nt && best1 < best) { mode = b1mode; best = best1; }
    if (b3a && b3b && best3 < best) { mode = smode; best = best3; }
    if (best6 < best) { mode = gmode; best = best6; }
    const bool streams = mode == 3 || mode == 4, groups = mode == 6 || mode == 7;
    f->tuned_mode[prec] = mode;
    f->tuned_nt[prec] = groups ? b6s : streams ? b3a : mode ? b1nt : b0nt;
    f->tuned_R[prec] = (streams || groups) ? sR : mode ? b1R : b0R;
    f->tuned_B[prec] = groups ? b6i : streams ? b3b : mode ? b1B : 1;
    f->tuned_ms[prec] = best;
    // drop the group tables unless a precision uses them
    const int other = f->tuned_mode[prec ^ 1];
    if (!groups && other != 6 && other != 7) {
        group_tables_free(&f->grp[0]);
        group_tables_free(&f->grp[1]);
    }
    if (mode != 1 && mode != 3 && mode != 6 && f->tbuf[prec]) {  // the product panels are not needed
        cudaFree(f->tbuf[prec]);
        f->tbuf[prec] = nullptr;
        f->mix_grid[prec] = 0;
    }
    if (!streams && !groups && f->sbuf[prec]) {  // the streaming scratch is not needed
        cudaFree(f->sbuf[prec]);
        f->sbuf[prec] = nullptr;
    }
    return JCI_OK;
}

void fci_tuning(const jci_space *s, int precision, int *mode, int *nt, int *R, int *B,
                float *ms) {
    const FciTables *f = s->dev ? s->dev->fci : nullptr;
    int p = precision == JCI_FP32 ? 1 : 0;
    *mode = f ? f->tuned_mode[p] : 0;
    *nt = f ? f->tuned_nt[p] : 0;
    *R = f ? f->tuned_R[p] : 0;
    *B = f ? f->tuned_B[p] : 0;
    *ms = f ? f->tuned_ms[p] : 0.f;
}

template <typename T>
static jci_status launch_fci(jci_space *s, int nvec, const T *V, T *S, long long ld,
                             cudaStream_t st) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    FciArgs<T> a;
    a.na = f->na; a.nb = f->nb; a.sa = f->sa; a.sb = f->sb; a.da = f->da; a.db = f->db;
    a.npair = f->npair;
    a.R = 1;
    a.do_as = 1;
    a.skip = d->sigma_skip;
    a.fsA = d->t[0].fsing; a.fsB = d->t[1].fsing;
    a.fpA = d->t[0].fspair; a.fpB = d->t[1].fspair;
    a.dJA = f->dblJ[0]; a.dJB = f->dblJ[1];
    if (prec == 0) {
        a.a1A = (const T *)f->d[0].a1T; a.a1B = (const T *)f->d[1].a1T;
        a.jA = (const T *)f->d[0].joccT; a.jB = (const T *)f->d[1].joccT;
        a.dHA = (const T *)f->d[0].dblH; a.dHB = (const T *)f->d[1].dblH;
        a.hd = (const T *)d->hd; a.m2 = (const T *)d->m2;
    } else {
        a.a1A = (const T *)f->f[0].a1T; a.a1B = (const T *)f->f[1].a1T;
        a.jA = (const T *)f->f[0].joccT; a.jB = (const T *)f->f[1].joccT;
        a.dHA = (const T *)f->f[0].dblH; a.dHB = (const T *)f->f[1].dblH;
        a.hd = (const T *)d->hdf; a.m2 = (const T *)d->m2f;
    }
    if (f->tuned_nt[prec] == 0) {
        jci_status r = autotune<T>(s, a, st);
        if (r) return r;
    }
    for (int c = 0; c < nvec; c++) {
        jci_status r = run_plan<T>(s, a, f->tuned_mode[prec], f->tuned_nt[prec],
                                   f->tuned_R[prec], f->tuned_B[prec], V + c * ld, S + c * ld,
                                   st);
        if (r) return r;
    }
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

jci_status fci_sigma(jci_space *s, int nvec, const void *v, void *sig, long long ld,
                     int precision, cudaStream_t st) {
    if (precision == JCI_FP32)
        return launch_fci<float>(s, nvec, (const float *)v, (float *)sig, ld, st);
    return launch_fci<double>(s, nvec, (const double *)v, (double *)sig, ld, st);
}

// Force a plan (modes as in run_plan) for tests and measurements; nt =
// threads per CTA of the row kernel (modes 3, 4: of the alpha pass, B =
// threads of the beta pass; modes 6, 7: of the beta-singles stream); R as
// the product kernel takes it.
jci_status fci_force_plan(jci_space *s, int precision, int mode, int nt, int R, int B) {
    FciTables *f = s->dev ? s->dev->fci : nullptr;
    if (!f) return JCI_ERR_STATE;
    int p = precision == JCI_FP32 ? 1 : 0;
    size_t w = p ? sizeof(float) : sizeof(double);
    if (mode == 6 || mode == 7) {
        bool ok = mode == 6 ? mixed_possible(f, w) && R >= 0 : ab_plan_possible(f, R, w);
        const bool beta_ok = nt == 0 ? hs_tables(s, s->dev->stream) == JCI_OK
                                     : stream_ok(f->na, nt) && stream_smem(0, f->sb, w) <= f->smem_max;
        if (!ok || !group_possible(f) || !beta_ok || B < 1 || B > 7) return JCI_ERR_ARG;
        if (B >= 5 && pair_tables(s, s->dev->stream) != JCI_OK) return JCI_ERR_ARG;
    } else if (mode == 3 || mode == 4) {
        bool ok = mode == 3 ? mixed_possible(f, w) && R >= 0 : ab_plan_possible(f, R, w);
        if (!ok || !stream_ok(f->nb, nt) || !stream_ok(f->na, B) ||
            stream_smem(f->da, 0, w) > f->smem_max || stream_smem(f->db, f->sb, w) > f->smem_max)
            return JCI_ERR_ARG;
    } else if (mode == 1 || mode == 2 || mode == 5) {
        bool ok = mode == 1   ? mixed_possible(f, w) && R >= 0
                  : mode == 2 ? mixed2_possible(f, w) && R >= 0
                              : ab_plan_possible(f, R, w);
        if (!ok || !rows_ok(f->nb, nt, B) || rows_smem(f->nb, f->npair, f->da, B, w) > f->smem_max)
            return JCI_ERR_ARG;
    } else {
        int items = (f->nb + nt - 1) / nt;
        if ((nt != 128 && nt != 256 && nt != 512 && nt != 1024) || items > 32 ||
            (nt == 1024 && items > 2))
            return JCI_ERR_ARG;
        if (R < 1 || fci_smem(f->nb, f->npair, R, w) > f->smem_max) return JCI_ERR_ARG;
    }
    if (mode == 4 || mode == 5 || mode == 7) {  // tables are built here, outside any capture
        AbTables *t = nullptr;
        jci_status r = ab_tables(s, ab_table_tx(R), s->dev->stream, &t);
        if (r) return r;
    }
    if (mode == 6 || mode == 7) {
        jci_status r = B >= 5 ? JCI_OK : group_tables(s, s->dev->stream);
        if (r) return r;
    }
    if ((mode == 1 || mode == 3 || mode == 6) && (R >= 128 || (R >= 64 && R - 64 >= 16)))
        return JCI_ERR_ARG;
    if ((mode == 1 || mode == 3 || mode == 6) && R >= 64) {  // compact panel tables
        jci_status r = compact_tables(s, s->dev->stream);
        if (r) return r == JCI_ERR_SPACE ? JCI_ERR_ARG : r;
    }
    if ((mode == 1 || mode == 3 || mode == 6) && R >= 16 && R < 32) {  // column-blocked lists
        AbTables *t = nullptr;
        jci_status r = ab_tables(s, kMixBlock / 4, s->dev->stream, &t);
        if (r) return r;
    }
    f->tuned_mode[p] = mode;
    f->tuned_nt[p] = nt;
    f->tuned_R[p] = R;
    f->tuned_B[p] = mode != 0 ? B : 1;
    f->tuned_ms[p] = 0.f;
    return JCI_OK;
}

// ---- allocation-free sigma ----------------------------------------------
//
// For callers that cannot allocate device memory while they run sigma: a
// driver that captures its whole iteration into a CUDA graph, a host that
// runs under a fixed device-memory budget, or an embedding application
// whose allocator forbids cudaMalloc / cudaFree after start-up.  The
// dense-product kernel's per-CTA panels come from this fixed, statically
// sized device array instead of a buffer allocated on first use; the
// tables built by jci_set_integrals are reused as they are.

constexpr size_t kNoAllocScratchBytes = 64ull << 20;  // 64 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
static void *g_noalloc_ptr[kMaxDevices];
static std::once_flag g_noalloc_once[kMaxDevices];
static cudaError_t g_noalloc_err[kMaxDevices];

// Device address of g_noalloc_scratch on device `dev`.  The host-side name
// is only a stand-in for the symbol, so the address is looked up once per
// device, with that device made current for the lookup (the caller's
// current device is restored afterwards), and cached.
static jci_status noalloc_scratch(int dev, void **out) {
    if (dev < 0 || dev >= kMaxDevices) return JCI_ERR_ARG;
    std::call_once(g_noalloc_once[dev], [dev]() {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e == cudaSuccess && prev != dev) e = cudaSetDevice(dev);
        if (e == cudaSuccess)
            e = cudaGetSymbolAddress(&g_noalloc_ptr[dev], g_noalloc_scratch);
        if (prev >= 0 && prev != dev) {
            cudaError_t e2 = cudaSetDevice(prev);
            if (e == cudaSuccess) e = e2;
        }
        g_noalloc_err[dev] = e;
    });
    if (g_noalloc_err[dev] != cudaSuccess)
        return cuda_fail(g_noalloc_err[dev], "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__,
                         __LINE__);
    *out = g_noalloc_ptr[dev];
    return JCI_OK;
}

template <typename T>
static jci_status sigma_noalloc(jci_space *s, const T *v, T *o, cudaStream_t st) {
    DeviceState *d = s->dev;
    FciTables *f = d->fci;
    const int prec = sizeof(T) == 8 ? 0 : 1;
    size_t w = sizeof(T);
    if (!mixed_possible(f, w)) return JCI_ERR_SPACE;
    FciArgs<T> a;
    a.na = f->na; a.nb = f->nb; a.sa = f->sa; a.sb = f->sb; a.da = f->da; a.db = f->db;
    a.npair = f->npair;
    a.R = 0;
    a.do_as = 0;
    a.skip = nullptr;
    a.fsA = d->t[0].fsing; a.fsB = d->t[1].fsing;
    a.fpA = d->t[0].fspair; a.fpB = d->t[1].fspair;
    a.dJA = f->dblJ[0]; a.dJB = f->dblJ[1];
    if (prec == 0) {
        a.a1A = (const T *)f->d[0].a1T; a.a1B = (const T *)f->d[1].a1T;
        a.jA = (const T *)f->d[0].joccT; a.jB = (const T *)f->d[1].joccT;
        a.dHA = (const T *)f->d[0].dblH; a.dHB = (const T *)f->d[1].dblH;
        a.hd = (const T *)d->hd; a.m2 = (const T *)d->m2;
    } else {
        a.a1A = (const T *)f->f[0].a1T; a.a1B = (const T *)f->f[1].a1T;
        a.jA = (const T *)f->f[0].joccT; a.jB = (const T *)f->f[1].joccT;
        a.dHA = (const T *)f->f[0].dblH; a.dHB = (const T *)f->f[1].dblH;
        a.hd = (const T *)d->hdf; a.m2 = (const T *)d->m2f;
    }
    MixArgs<T> m;
    m.na = a.na; m.nb = a.nb; m.nbp = (a.nb + kMixCols - 1) / kMixCols * kMixCols;
    m.sa = a.sa; m.sb = a.sb; m.npair = a.npair; m.mrows = a.npair + 1;
    m.fsA = a.fsA; m.fsB = a.fsB; m.fpA = a.fpA; m.fpB = a.fpB;
    m.a1A = a.a1A; m.m2 = a.m2; m.occB = d->t[1].occ;
    m.skip = nullptr;
    size_t panel = (size_t)m.mrows * m.nbp * w;
    if (panel > kNoAllocScratchBytes) return JCI_ERR_SPACE;  // one row's panel must fit
    int TM = (m.mrows + 15) / 16;
    MixKernel<T> kern = mixed_kernel<T>(TM);
    if (!kern) return JCI_ERR_SPACE;
    void *scratch = nullptr;
    jci_status r = noalloc_scratch(d->device, &scratch);
    if (r) return r;
    // Row kernel k_sigma_fci.  The tuned thread count is a k_sigma_fci shape
    // only when the autotuner picked mode 0; every other mode's count belongs
    // to another kernel, so a fixed shape is used then.  Either way the
    // shape is checked as fci_force_plan checks mode 0 before anything runs.
    int nt = f->tuned_mode[prec] == 0 && f->tuned_nt[prec] ? f->tuned_nt[prec]
                                                           : (a.nb > 2048 ? 512 : 256);
    int items = (a.nb + nt - 1) / nt;
    if ((nt != 128 && nt != 256 && nt != 512 && nt != 1024) || items > 32 ||
        (nt == 1024 && items > 2))
        return JCI_ERR_SPACE;
    size_t row_smem = fci_smem(a.nb, a.npair, 0, w);
    if (row_smem > f->smem_max) return JCI_ERR_SPACE;
    if ((r = launch_one<T>(a, nt, row_smem, a.na, v, o, st))) return r;
    JCI_CUDA(cudaGetLastError());  // the product adds into the row kernel's output
    size_t smem = mix_smem(m.sa, TM, w);
    JCI_CUDA(smem_optin(kern));
    int occ = 0, nsm = 0;
    JCI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kMixThreads, smem));
    JCI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d->device));
    int grid = (int)std::min<size_t>(kNoAllocScratchBytes / panel,
                                     (size_t)nsm * std::max(occ, 1));
    grid = std::max(1, std::min(grid, m.na));
    kern<<<grid, kMixThreads, smem, st>>>(m, v, o, (T *)scratch);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

jci_status fci_sigma_noalloc(jci_space *s, const void *v, void *o, int precision,
                             cudaStream_t st) {
    if (!s->dev || !s->dev->fci || !s->dev->single_group) return JCI_ERR_SPACE;
    if (precision == JCI_FP32) return sigma_noalloc<float>(s, (const float *)v, (float *)o, st);
    return sigma_noalloc<double>(s, (const double *)v, (double *)o, st);
}

size_t fci_noalloc_scratch_bytes() { return kNoAllocScratchBytes; }

}  // namespace jci
