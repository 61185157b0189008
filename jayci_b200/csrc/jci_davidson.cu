// jci_davidson.cu -- Davidson eigensolver with every vector resident on the
// device (the reference keeps V, C, N, R, X, D in Global Arrays,
// pdavidson.c:111-135).
//
// Two schedules share the kernels below:
//  * block = 0: the reference's root-sequential algorithm (pdavidson.c:39):
//    one correction vector per iteration for the current root, classical
//    Gram-Schmidt in one pass (:4086), collapse to krymin Ritz vectors when
//    the space reaches krymax (:4821).  The subspace matrix is V_i . C_j for
//    i >= j (make_subspacehmat_ga :4053 read through dsyevr's upper
//    triangle), the residual r = sum_i y_i (c_i - theta v_i) (:3802), the
//    correction t = r / (theta - D) (:3773).  After a collapse every sigma
//    vector is recomputed, as in the reference.
//  * block = 1: block Davidson over all unconverged roots (one correction
//    per root per iteration, two Gram-Schmidt passes), so a sigma launch
//    processes several vectors and every root converges together.
// Precision: JCI_FP64, or JCI_MIXED = FP32 sigma (FP32 storage and
// accumulation) until the residual norms drop below switch_tol, then the
// basis is collapsed to the krymin lowest Ritz vectors and their sigma
// vectors are recomputed in FP64.  With block = 0 the mixed schedule takes
// every root below switch_tol before switching (two root-sequential
// phases), rotates sigma vectors with the Ritz coefficients at a collapse
// instead of recomputing them, and refines after the switch with FP32
// sigma for the new correction vectors and an FP64 sigma of the current
// root's Ritz vector at every stop (run_sequential); with block = 1 the
// iterations after the switch run in FP64.
// Basis vectors, Gram-Schmidt, residuals, the Hdiag preconditioner, the
// Rayleigh-Ritz eigensolve and the energies are FP64 throughout.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "jci_kernels.cuh"

namespace jci {

constexpr int kMaxKry = 64;
constexpr int kDotBlocks = 4 * 148;  // upper bound of the product grids (4 per SM)
constexpr int kHist = kMaxKry + 2;

// Control block of a graph-captured iteration of the root-sequential
// schedule (device memory).  The host writes it before a batch of graph
// launches and reads it afterwards; every kernel of the captured iteration
// takes its sizes from it and returns at once once stop is set, so launches
// after the stop cost a few microseconds and no sigma work.
struct DavCtl {
    int ckdim;     // basis vectors
    int croot;     // current root, 0-based
    int stop;      // 0 running, 1 residual below tol, 2 basis full, 3 eigensolve failed
    int iters;     // vectors added since the host wrote the block
    int nhist;     // residual tests recorded in the history
    int pad;
    double tol;    // residual-norm tolerance of the current phase
    double theta;  // Ritz value of the current root
};

struct DavHist {
    int root, ckdim;
    double theta, rnorm;
};

struct DavidsonBuffers {
    long long ld = 0;
    int cap = 0;             // vectors allocated in V and C
    double *V = nullptr, *C = nullptr, *X = nullptr, *Y2 = nullptr;
    double *r = nullptr, *t = nullptr;
    float *v32 = nullptr, *s32 = nullptr;
    int cap32 = 0;
    double *partial = nullptr;   // kDotBlocks x 64 x 16 (k_gram block partials)
    double *dots = nullptr;      // 64 x 16 (k_gram results)
    double *G = nullptr, *evec = nullptr, *eval = nullptr;
    double *coef = nullptr;      // 2 x kMaxKry x kMaxKry
    // graph-captured iterations
    DavCtl *ctl = nullptr;
    DavHist *hist = nullptr;     // kHist
    double *cnew = nullptr;      // sigma of the new basis vector (ld)
    int *info = nullptr;         // status word of k_jacobi
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // FP64, FP32 sigma
    int gkmax[2] = {0, 0};
    int gplan[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
};

static void drop_graphs(DavidsonBuffers *b) {
    for (int i = 0; i < 2; i++) {
        if (b->gexec[i]) cudaGraphExecDestroy(b->gexec[i]);
        b->gexec[i] = nullptr;
        b->gkmax[i] = 0;
    }
}

void davidson_free(DeviceState *d) {
    DavidsonBuffers *b = d->dav;
    if (!b) return;
    drop_graphs(b);
    void *p[] = {b->V, b->C, b->X, b->Y2, b->r, b->t, b->v32, b->s32, b->partial,
                 b->dots, b->G, b->evec, b->eval, b->coef, b->ctl, b->hist, b->cnew,
                 b->info};
    for (void *q : p) cudaFree(q);
    delete b;
    d->dav = nullptr;
}

// ---- kernels -------------------------------------------------------------

// Tall-skinny products G = X^T Y of basis panels (X: m <= 64 vectors, Y:
// p <= 16 vectors, each n long, vector-major with leading dimension ld) on
// the FP64 tensor cores: mma.sync m8n8k4 with A = 8 vectors of X x 4
// elements, B = the same 4 elements of 8 vectors of Y.  Lane (g = lane/4,
// t = lane%4) loads the element pair k+2t, k+2t+1 of vector 8a+g (A) and
// 8b+g (B) with one 16-byte load and feeds the two elements to two MMAs, so
// each load instruction reads 64 contiguous bytes of eight vectors, and the
// eight warps of a block together read 512 contiguous bytes.  The warps' 8x8
// tiles are summed in warp order in shared memory, the block partials in
// block order by k_gram_finish, so the result is bitwise reproducible.
constexpr int kGramRows = 64, kGramCols = 16;

__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// elements k, k+1 of row r (k even, r 16-byte aligned); zero past hi
__device__ __forceinline__ double2 load_pair(const double *__restrict__ r, long long k,
                                             long long hi, bool valid) {
    if (!valid || k >= hi) return make_double2(0.0, 0.0);
    if (k + 1 < hi) return *reinterpret_cast<const double2 *>(r + k);
    return make_double2(r[k], 0.0);
}

// Row count taken from a graph-captured iteration's control block: m =
// *mdev + madd (must stay <= 8 MT); kernels return at once when *stop != 0.
struct GramDev {
    const int *stop = nullptr;
    const int *mdev = nullptr;
    int madd = 0;
};

// partial[blk][i*p + j] = sum over this block's slice of X_i . Y_j
template <int MT, int PT>
__global__ void __launch_bounds__(256)
    k_gram(const double *__restrict__ X, int m, const double *__restrict__ Y, int p,
           long long ld, long long n, long long chunk, double *__restrict__ partial,
           GramDev gd) {
    if (gd.stop && *gd.stop) return;
    if (gd.mdev) m = *gd.mdev + gd.madd;
    __shared__ double red[MT * 8][PT * 8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const long long lo = (long long)blockIdx.x * chunk, hi = min(n, lo + chunk);
    const double *xr[MT], *yr[PT];
    bool xv[MT], yv[PT];
#pragma unroll
    for (int a = 0; a < MT; a++) {
        xv[a] = 8 * a + g < m;
        xr[a] = X + (long long)(xv[a] ? 8 * a + g : 0) * ld;
    }
#pragma unroll
    for (int b = 0; b < PT; b++) {
        yv[b] = 8 * b + g < p;
        yr[b] = Y + (long long)(yv[b] ? 8 * b + g : 0) * ld;
    }
    double acc[MT][PT][2];
#pragma unroll
    for (int a = 0; a < MT; a++)
#pragma unroll
        for (int b = 0; b < PT; b++) acc[a][b][0] = acc[a][b][1] = 0.0;
    // The slice is cut into 8-element groups; group g goes to warp g % 8
    // and each warp takes its groups in ascending order, whatever U (the
    // groups in flight per step), so the summation order and the result are
    // the same for every kernel shape.
    constexpr int U = MT <= 2 ? 4 : (MT <= 4 ? 2 : 1);
    for (long long g0 = warp; lo + 8 * g0 < hi; g0 += 8 * U) {
        double2 av[U][MT], bv[U][PT];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const long long k = lo + 8 * (g0 + 8 * u) + 2 * t;
#pragma unroll
            for (int a = 0; a < MT; a++) av[u][a] = load_pair(xr[a], k, hi, xv[a]);
#pragma unroll
            for (int b = 0; b < PT; b++) bv[u][b] = load_pair(yr[b], k, hi, yv[b]);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int a = 0; a < MT; a++)
#pragma unroll
                for (int b = 0; b < PT; b++) {
                    dmma_8x8x4(acc[a][b], av[u][a].x, bv[u][b].x);
                    dmma_8x8x4(acc[a][b], av[u][a].y, bv[u][b].y);
                }
    }
    // accumulator layout: lane holds row g, columns 2t and 2t+1 of each tile
    for (int w = 0; w < 8; w++) {
        if (warp == w) {
#pragma unroll
            for (int a = 0; a < MT; a++)
#pragma unroll
                for (int b = 0; b < PT; b++)
#pragma unroll
                    for (int i = 0; i < 2; i++) {
                        double &r = red[8 * a + g][8 * b + 2 * t + i];
                        r = w ? r + acc[a][b][i] : acc[a][b][i];
                    }
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < m * p; e += blockDim.x)
        partial[(long long)blockIdx.x * kGramRows * kGramCols + e] = red[e / p][e % p];
}

// G = X^T y for one vector y (p = 1: the basis products of every iteration)
// on the FP64 FMA pipes: an m8n8k4 product with one valid column would do
// eight times the arithmetic, and at 48 rows that padding costs as much time
// as the loads.  Row i belongs to warp i % 8; every warp reads the whole
// slice of y (from L1 after the first warp) and of its rows, lane l taking
// the element pairs lo + 64 j + 2 l in ascending j, U pairs per step, so a
// thread keeps MT x U 16-byte loads in flight.  A row's sum runs in the same
// order whatever MT and U, so host-driven and graph-captured iterations
// (different MT) agree bitwise.  Block partial of row i in partial[blk][i],
// summed in block order by k_gram_finish.
template <int MT>
__global__ void __launch_bounds__(256)
    k_gram_vec(const double *__restrict__ X, int m, const double *__restrict__ y, long long ld,
               long long n, long long chunk, double *__restrict__ partial, GramDev gd) {
    if (gd.stop && *gd.stop) return;
    if (gd.mdev) m = *gd.mdev + gd.madd;
    constexpr int U = MT <= 2 ? 8 : (MT <= 4 ? 4 : 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long lo = (long long)blockIdx.x * chunk, hi = min(n, lo + chunk);
    const double *xr[MT];
    bool xv[MT];
#pragma unroll
    for (int a = 0; a < MT; a++) {
        xv[a] = 8 * a + warp < m;
        xr[a] = X + (long long)(xv[a] ? 8 * a + warp : 0) * ld;
    }
    double acc[MT];
#pragma unroll
    for (int a = 0; a < MT; a++) acc[a] = 0.0;
    for (long long k0 = lo + 2 * lane; k0 < hi; k0 += 64 * U) {
        double2 yv[U], xvv[U][MT];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const long long k = k0 + 64 * u;
            yv[u] = load_pair(y, k, hi, true);
#pragma unroll
            for (int a = 0; a < MT; a++) xvv[u][a] = load_pair(xr[a], k, hi, xv[a]);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int a = 0; a < MT; a++) {
                acc[a] = fma(xvv[u][a].x, yv[u].x, acc[a]);
                acc[a] = fma(xvv[u][a].y, yv[u].y, acc[a]);
            }
    }
#pragma unroll
    for (int a = 0; a < MT; a++) {
        double s = acc[a];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0 && xv[a])
            partial[(long long)blockIdx.x * kGramRows * kGramCols + 8 * a + warp] = s;
    }
}

using GramVecKernel = void (*)(const double *, int, const double *, long long, long long,
                               long long, double *, GramDev);

static GramVecKernel gram_vec_kernel(int mt) {
    switch (mt) {
        case 1: return k_gram_vec<1>;
        case 2: return k_gram_vec<2>;
        case 3: return k_gram_vec<3>;
        case 4: return k_gram_vec<4>;
        case 5: return k_gram_vec<5>;
        case 6: return k_gram_vec<6>;
        case 7: return k_gram_vec<7>;
        default: return k_gram_vec<8>;
    }
}

// Single dot product x . y (norms): every lane loads, block partial in
// partial[blk][0], summed in block order by k_gram_finish.
__global__ void __launch_bounds__(256)
    k_dot(const double *__restrict__ x, const double *__restrict__ y, long long n,
          long long chunk, double *__restrict__ partial, GramDev gd) {
    if (gd.stop && *gd.stop) return;
    __shared__ double red[8];
    const long long lo = (long long)blockIdx.x * chunk, hi = min(n, lo + chunk);
    double s = 0.0;
    for (long long k = lo + threadIdx.x; k < hi; k += 256) s += x[k] * y[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += red[w];
        partial[(long long)blockIdx.x * kGramRows * kGramCols] = t;
    }
}

// out[e] = sum_b partial[b][e] in a fixed order (bitwise reproducible).
__global__ void k_gram_finish(const double *__restrict__ partial, int nb, int mp, double *out,
                              GramDev gd, int p) {
    if (gd.stop && *gd.stop) return;
    if (gd.mdev) mp = (*gd.mdev + gd.madd) * p;
    const int e = blockIdx.x;
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) s += partial[(long long)b * kGramRows * kGramCols + e];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0 && e < mp) out[e] = s;
}

using GramKernel = void (*)(const double *, int, const double *, int, long long, long long,
                            long long, double *, GramDev);

template <int MT>
static GramKernel gram_kernel_p(int pt) {
    return pt == 1 ? k_gram<MT, 1> : k_gram<MT, 2>;
}

static GramKernel gram_kernel(int mt, int pt) {
    switch (mt) {
        case 1: return gram_kernel_p<1>(pt);
        case 2: return gram_kernel_p<2>(pt);
        case 3: return gram_kernel_p<3>(pt);
        case 4: return gram_kernel_p<4>(pt);
        case 5: return gram_kernel_p<5>(pt);
        case 6: return gram_kernel_p<6>(pt);
        case 7: return gram_kernel_p<7>(pt);
        default: return gram_kernel_p<8>(pt);
    }
}

// out[k] = sum_i a[i] X_i[k] + sum_i b[i] Y_i[k]   (coefficients on device)
// (with ctl: mx = my = ctl->ckdim, nothing when ctl->stop)
__global__ void k_lincomb(double *__restrict__ out, long long n, long long ld,
                          const double *__restrict__ X, const double *__restrict__ a, int mx,
                          const double *__restrict__ Y, const double *__restrict__ b, int my,
                          const DavCtl *ctl) {
    if (ctl) {
        if (ctl->stop) return;
        mx = my = ctl->ckdim;
    }
    __shared__ double ca[kMaxKry], cb[kMaxKry];
    for (int i = threadIdx.x; i < mx; i += blockDim.x) ca[i] = a[i];
    for (int i = threadIdx.x; i < my; i += blockDim.x) cb[i] = b[i];
    __syncthreads();
    // element pairs with 16-byte loads (ld is a multiple of 32 and the panels
    // 256-byte aligned, so every pair is aligned); the same sums, in the same
    // order, as one element at a time
    const long long n2 = n / 2;
    for (long long k2 = (long long)blockIdx.x * blockDim.x + threadIdx.x; k2 < n2;
         k2 += (long long)gridDim.x * blockDim.x) {
        const long long k = 2 * k2;
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
        for (int i = 0; i < mx; i++) {
            const double2 x = *reinterpret_cast<const double2 *>(X + i * ld + k);
            s0 += ca[i] * x.x;
            s1 += ca[i] * x.y;
        }
#pragma unroll 4
        for (int i = 0; i < my; i++) {
            const double2 y = *reinterpret_cast<const double2 *>(Y + i * ld + k);
            s0 += cb[i] * y.x;
            s1 += cb[i] * y.y;
        }
        *reinterpret_cast<double2 *>(out + k) = make_double2(s0, s1);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long long k = n - 1;
        double s = 0.0;
        for (int i = 0; i < mx; i++) s += ca[i] * X[i * ld + k];
        for (int i = 0; i < my; i++) s += cb[i] * Y[i * ld + k];
        out[k] = s;
    }
}

// t -= sum_i ov[i] X_i ; used by classical Gram-Schmidt
__global__ void k_orth_update(double *__restrict__ t, long long n, long long ld,
                              const double *__restrict__ X, const double *__restrict__ ov,
                              int m, const DavCtl *ctl) {
    if (ctl) {
        if (ctl->stop) return;
        m = ctl->ckdim;
    }
    __shared__ double c[kMaxKry];
    for (int i = threadIdx.x; i < m; i += blockDim.x) c[i] = ov[i];
    __syncthreads();
    const long long n2 = n / 2;  // element pairs, 16-byte loads (as k_lincomb)
    for (long long k2 = (long long)blockIdx.x * blockDim.x + threadIdx.x; k2 < n2;
         k2 += (long long)gridDim.x * blockDim.x) {
        const long long k = 2 * k2;
        double2 s = *reinterpret_cast<const double2 *>(t + k);
#pragma unroll 8
        for (int i = 0; i < m; i++) {
            const double2 x = *reinterpret_cast<const double2 *>(X + i * ld + k);
            s.x -= c[i] * x.x;
            s.y -= c[i] * x.y;
        }
        *reinterpret_cast<double2 *>(t + k) = s;
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long long k = n - 1;
        double s = t[k];
        for (int i = 0; i < m; i++) s -= c[i] * X[i * ld + k];
        t[k] = s;
    }
}

// t = r / (theta - D)   (generate_newvector, pdavidson.c:3773)
__global__ void k_precond(const double *__restrict__ r, const double *__restrict__ D,
                          double theta, double *__restrict__ t, long long n,
                          const DavCtl *ctl) {
    if (ctl) {
        if (ctl->stop) return;
        theta = ctl->theta;
    }
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        double den = theta - D[k];
        // the reference divides without a guard; an exact zero would give inf
        if (fabs(den) < 1e-14) den = den < 0 ? -1e-14 : 1e-14;
        t[k] = r[k] / den;
    }
}

// x *= 1 / sqrt(*nrm2)
__global__ void k_normalize(double *__restrict__ x, long long n, const double *__restrict__ nrm2,
                            const int *stop) {
    if (stop && *stop) return;
    double s = 1.0 / sqrt(*nrm2);
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        x[k] *= s;
}

__global__ void k_d2f(const double *__restrict__ in, float *__restrict__ out, long long n,
                      long long ldi, long long ldo, int m, const int *stop) {
    if (stop && *stop) return;
    for (int c = 0; c < m; c++)
        for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
             k += (long long)gridDim.x * blockDim.x)
            out[c * ldo + k] = (float)in[c * ldi + k];
}

__global__ void k_f2d(const float *__restrict__ in, double *__restrict__ out, long long n,
                      long long ldi, long long ldo, int m, const int *stop) {
    if (stop && *stop) return;
    for (int c = 0; c < m; c++)
        for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
             k += (long long)gridDim.x * blockDim.x)
            out[c * ldo + k] = (double)in[c * ldi + k];
}

// Jacobi eigensolve of the m x m symmetric matrix held in the lower
// triangle of G (G[i*ldg + j], i >= j), one CTA of kJacobiThreads threads.
// Parallel cyclic Jacobi: a sweep is m'-1 rounds (m' = m rounded up to
// even) of m'/2 disjoint rotations in round-robin order (one index fixed,
// the others rotating), so a round applies J^T A J for all its pairs at
// once: angles, then the column updates (with those of the eigenvector
// matrix), then the row updates; pair j goes to warp j % 8, element k to
// lane k % 32.  Each rotation annihilates A[p][q] with the classic angle
// t = sign(th) / (|th| + sqrt(th^2 + 1)), th = (Aqq - App) / 2Apq.
// Converged when the sum of squared off-diagonal entries is below 1e-30 of
// the diagonal's.  Eigenvalues ascending in w (equal values keep their
// index order); eigenvector k in Y[k*ldg + .], sign fixed so that its
// largest-magnitude component is positive.  info = number of sweeps, or -1
// if not converged in 60.
//
// With arrow set, w / Y hold on entry the eigenpairs of the leading
// (m-1) x (m-1) block of G (the previous Rayleigh-Ritz step, before a row
// was appended).  The sweeps then start from Q^T G Q with Q = diag(Y^T, 1):
// diag(w) bordered by the new row Y g and G[m-1][m-1] (an arrowhead matrix),
// with the eigenvector matrix started at Q, which takes a few sweeps instead
// of a full diagonalisation.
constexpr int kJacobiThreads = 256;

__global__ void __launch_bounds__(kJacobiThreads)
    k_jacobi(const double *__restrict__ G, int m, int ldg, double *w, double *Y, int *info,
             const DavCtl *ctl, int arrow) {
    if (ctl) {
        if (ctl->stop) return;
        m = ctl->ckdim;
    }
    extern __shared__ double sm[];
    const int st = m + 1;
    double *A = sm;                 // m x (m+1)
    double *Vm = sm + m * st;       // m x (m+1)
    __shared__ double rc[kMaxKry / 2], rs[kMaxKry / 2];
    __shared__ int rp[kMaxKry / 2], rq[kMaxKry / 2];
    __shared__ double red_off[kJacobiThreads / 32], red_dia[kJacobiThreads / 32];
    __shared__ int s_conv;
    __shared__ int order[kMaxKry];
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31;
    const int nwarp = nt >> 5;
    if (arrow && m > 1) {
        const int p = m - 1;
        for (int i = tid; i < m * m; i += nt) {
            int r = i / m, c = i % m;
            A[r * st + c] = r == c && r < p ? w[r] : 0.0;
            Vm[r * st + c] = r < p && c < p ? Y[c * ldg + r] : (r == c ? 1.0 : 0.0);
        }
        __syncthreads();
        for (int k = tid; k < p; k += nt) {
            double x = 0.0;
            for (int i = 0; i < p; i++) x += Y[k * ldg + i] * G[p * ldg + i];
            A[k * st + p] = x;
            A[p * st + k] = x;
        }
        if (tid == 0) A[p * st + p] = G[p * ldg + p];
    } else {
        for (int i = tid; i < m * m; i += nt) {
            int r = i / m, c = i % m;
            A[r * st + c] = r >= c ? G[r * ldg + c] : G[c * ldg + r];
            Vm[r * st + c] = r == c ? 1.0 : 0.0;
        }
    }
    __syncthreads();
    const int me = m + (m & 1), npr = me / 2;
    int sweep = 0, conv = 0;
    for (; sweep < 60; sweep++) {
        double off = 0.0, dia = 0.0;
        for (int i = tid; i < m * m; i += nt) {
            int r = i / m, c = i % m;
            double x = A[r * st + c];
            if (r != c) off += x * x;
            else dia += x * x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            dia += __shfl_xor_sync(0xffffffffu, dia, o);
        }
        if (lane == 0) {
            red_off[warp] = off;
            red_dia[warp] = dia;
        }
        __syncthreads();
        if (tid == 0) {
            double so = 0.0, sd = 0.0;
            for (int k = 0; k < nwarp; k++) {
                so += red_off[k];
                sd += red_dia[k];
            }
            s_conv = so <= 1e-30 * fmax(sd, 1e-300);
        }
        __syncthreads();
        if (s_conv) {
            conv = 1;
            break;
        }
        for (int round = 0; round < me - 1; round++) {
            if (tid < npr) {
                // circle method: position 0 fixed, positions 1..me-1 rotate
                int a = tid, b = me - 1 - tid;
                int p = a == 0 ? 0 : (a - 1 + round) % (me - 1) + 1;
                int q = b == 0 ? 0 : (b - 1 + round) % (me - 1) + 1;
                if (p > q) {
                    int x = p;
                    p = q;
                    q = x;
                }
                double c = 1.0, sn = 0.0;
                if (q < m) {
                    double apq = A[p * st + q], app = A[p * st + p], aqq = A[q * st + q];
                    if (!(fabs(apq) <= 1e-300 || fabs(apq) <= 1e-18 * sqrt(fabs(app * aqq)))) {
                        double th = (aqq - app) / (2.0 * apq);
                        double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        sn = t * c;
                    }
                }
                rp[tid] = p;
                rq[tid] = q < m ? q : p;
                rc[tid] = c;
                rs[tid] = sn;
            }
            __syncthreads();
            // columns p, q of A and of the eigenvector matrix
            for (int j = warp; j < npr; j += nwarp) {
                const double c = rc[j], sn = rs[j];
                if (sn == 0.0) continue;
                const int p = rp[j], q = rq[j];
                for (int k = lane; k < m; k += 32) {
                    double akp = A[k * st + p], akq = A[k * st + q];
                    A[k * st + p] = c * akp - sn * akq;
                    A[k * st + q] = sn * akp + c * akq;
                    double vkp = Vm[k * st + p], vkq = Vm[k * st + q];
                    Vm[k * st + p] = c * vkp - sn * vkq;
                    Vm[k * st + q] = sn * vkp + c * vkq;
                }
            }
            __syncthreads();
            // rows p, q of A
            for (int j = warp; j < npr; j += nwarp) {
                const double c = rc[j], sn = rs[j];
                if (sn == 0.0) continue;
                const int p = rp[j], q = rq[j];
                for (int k = lane; k < m; k += 32) {
                    double apk = A[p * st + k], aqk = A[q * st + k];
                    A[p * st + k] = c * apk - sn * aqk;
                    A[q * st + k] = sn * apk + c * aqk;
                }
            }
            __syncthreads();
        }
    }
    // eigenvalue order: rank of each diagonal entry, ties by index
    for (int i = tid; i < m; i += nt) {
        double x = A[i * st + i];
        int r = 0;
        for (int j = 0; j < m; j++) {
            double y = A[j * st + j];
            r += (y < x) || (y == x && j < i);
        }
        order[r] = i;
    }
    __syncthreads();
    for (int k = tid; k < m; k += nt) {
        int c = order[k];
        w[k] = A[c * st + c];
        double big = 0.0;
        int bi = 0;
        for (int i = 0; i < m; i++)
            if (fabs(Vm[i * st + c]) > big + 1e-14) {
                big = fabs(Vm[i * st + c]);
                bi = i;
            }
        double sg = Vm[bi * st + c] < 0 ? -1.0 : 1.0;
        for (int i = 0; i < m; i++) Y[k * ldg + i] = sg * Vm[i * st + c];
    }
    if (tid == 0) *info = conv ? sweep : -1;
}

// ---- kernels of a graph-captured iteration (one CTA, except k_it_store) ----

// residual coefficients of the current root: r = C y - theta V y
__global__ void k_it_begin(DavCtl *c, const double *__restrict__ eval,
                           const double *__restrict__ evec, double *coef) {
    if (c->stop) return;
    const int k = c->croot, m = c->ckdim;
    const double th = eval[k];
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        double y = evec[k * kMaxKry + i];
        coef[i] = y;
        coef[kMaxKry + i] = -th * y;
    }
    if (threadIdx.x == 0) c->theta = th;
}

// residual-norm test; the iteration is recorded for the host's log
__global__ void k_it_check(DavCtl *c, const double *__restrict__ rn2, DavHist *hist) {
    if (c->stop) return;
    const double rn = sqrt(*rn2);
    const int h = c->nhist;
    if (h < kHist) hist[h] = DavHist{c->croot, c->ckdim, c->theta, rn};
    c->nhist = h + 1;
    if (rn < c->tol) c->stop = 1;
}

// dst + (ckdim + off) * ld  <-  src
__global__ void k_it_store(double *__restrict__ dst, long long ld, int off,
                           const double *__restrict__ src, long long n, const DavCtl *c) {
    if (c->stop) return;
    double *d = dst + (long long)(c->ckdim + off) * ld;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        d[k] = src[k];
}

// new row G[ckdim][0..ckdim] of the subspace matrix; the basis grows by one
__global__ void k_it_append(DavCtl *c, const double *__restrict__ dots, double *G) {
    if (c->stop) return;
    const int m = c->ckdim;
    for (int j = threadIdx.x; j <= m; j += blockDim.x) G[m * kMaxKry + j] = dots[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        c->ckdim = m + 1;
        c->iters++;
    }
}

__global__ void k_it_end(DavCtl *c, const int *__restrict__ info, int kmax) {
    if (c->stop) return;
    if (*info < 0) c->stop = 3;
    else if (c->ckdim >= kmax) c->stop = 2;
}

// ---- host driver ---------------------------------------------------------

static unsigned grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (unsigned)std::max(1LL, std::min(g, 148LL * 8));
}

struct Ctx {
    jci_space *s;
    DeviceState *d;
    DavidsonBuffers *b;
    cudaStream_t st;
    long long n, ld;
    int *d_info = nullptr;
    double sigma_ms = 0.0;
    double ms_per_vec[2] = {0.0, 0.0};  // last measured sigma time per vector (FP64, FP32)
    int sigma_calls = 0;
    long long sigma_vecs = 0;
    int fp32_vecs = 0;
};

static jci_status ensure_buffers(Ctx &c, int cap, bool mixed, int maxnew) {
    DeviceState *d = c.d;
    if (!d->dav) d->dav = new DavidsonBuffers();
    DavidsonBuffers *b = d->dav;
    c.b = b;
    long long ld = (c.n + 31) / 32 * 32;
    if (b->ld != ld || b->cap < cap) {
        drop_graphs(b);
        void *p[] = {b->V, b->C, b->X, b->r, b->t, b->cnew};
        for (void *q : p) cudaFree(q);
        b->ld = ld;
        b->cap = cap;
        JCI_CUDA(cudaMalloc(&b->V, (size_t)cap * ld * sizeof(double)));
        JCI_CUDA(cudaMalloc(&b->C, (size_t)cap * ld * sizeof(double)));
        JCI_CUDA(cudaMalloc(&b->X, (size_t)cap * ld * sizeof(double)));
        JCI_CUDA(cudaMalloc(&b->r, (size_t)ld * sizeof(double)));
        JCI_CUDA(cudaMalloc(&b->t, (size_t)ld * sizeof(double)));
        JCI_CUDA(cudaMalloc(&b->cnew, (size_t)ld * sizeof(double)));
        if (!b->partial) {
            JCI_CUDA(cudaMalloc(&b->ctl, sizeof(DavCtl)));
            JCI_CUDA(cudaMalloc(&b->hist, kHist * sizeof(DavHist)));
            JCI_CUDA(cudaMalloc(&b->info, sizeof(int)));
            JCI_CUDA(cudaMalloc(&b->partial,
                                (size_t)kDotBlocks * kGramRows * kGramCols * sizeof(double)));
            JCI_CUDA(cudaMalloc(&b->dots, kGramRows * kGramCols * sizeof(double)));
            JCI_CUDA(cudaMalloc(&b->G, kMaxKry * kMaxKry * sizeof(double)));
            JCI_CUDA(cudaMalloc(&b->evec, kMaxKry * kMaxKry * sizeof(double)));
            JCI_CUDA(cudaMalloc(&b->eval, kMaxKry * sizeof(double)));
            JCI_CUDA(cudaMalloc(&b->coef, 2 * kMaxKry * kMaxKry * sizeof(double)));
        }
    }
    if (mixed && (b->cap32 < maxnew || !b->v32)) {
        drop_graphs(b);
        cudaFree(b->v32);
        cudaFree(b->s32);
        b->cap32 = maxnew;
        JCI_CUDA(cudaMalloc(&b->v32, (size_t)maxnew * ld * sizeof(float)));
        JCI_CUDA(cudaMalloc(&b->s32, (size_t)maxnew * ld * sizeof(float)));
    }
    c.ld = ld;
    JCI_CUDA(cudaMemsetAsync(b->V, 0, (size_t)cap * ld * sizeof(double), c.st));
    JCI_CUDA(cudaMemsetAsync(b->C, 0, (size_t)cap * ld * sizeof(double), c.st));
    return JCI_OK;
}

// C[i0 .. i0+m) = H V[i0 .. i0+m) in the requested precision
static jci_status sigma_block(Ctx &c, int i0, int m, bool fp32) {
    DavidsonBuffers *b = c.b;
    cudaEvent_t e0 = c.d->ev0, e1 = c.d->ev1;
    jci_status r;
    double ms_call = 0.0;
    if (fp32) {
        for (int k0 = 0; k0 < m; k0 += b->cap32) {
            int mm = std::min(b->cap32, m - k0);
            k_d2f<<<grid_for(c.n), 256, 0, c.st>>>(b->V + (i0 + k0) * c.ld, b->v32, c.n, c.ld,
                                                   c.ld, mm, nullptr);
            if ((r = device_sigma(c.s, mm, b->v32, b->s32, c.ld, JCI_FP32, c.st))) return r;
            float ms = 0.f;
            JCI_CUDA(cudaEventSynchronize(e1));
            JCI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms_call += ms;
            k_f2d<<<grid_for(c.n), 256, 0, c.st>>>(b->s32, b->C + (i0 + k0) * c.ld, c.n, c.ld,
                                                   c.ld, mm, nullptr);
        }
        c.fp32_vecs += m;
    } else {
        if ((r = device_sigma(c.s, m, b->V + i0 * c.ld, b->C + i0 * c.ld, c.ld, JCI_FP64,
                              c.st)))
            return r;
        float ms = 0.f;
        JCI_CUDA(cudaEventSynchronize(e1));
        JCI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        ms_call = ms;
    }
    c.sigma_ms += ms_call;
    c.ms_per_vec[fp32 ? 1 : 0] = ms_call / m;
    c.sigma_calls++;
    c.sigma_vecs += m;
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

// out[i*p + j] = X_i . Y_j on the device (i < m <= 64, j < p <= 16)
static jci_status gram(Ctx &c, const double *X, int m, const double *Y, int p, double *out,
                       GramDev gd = GramDev()) {
    if (m < 1 || m > kGramRows || p < 1 || p > kGramCols) return JCI_ERR_ARG;
    const bool dot = m == 1 && p == 1 && !gd.mdev;
    // a fixed partition (kDotBlocks slices): the summation order, and so
    // every bit of the result, is the same for every kernel shape and for
    // graph-captured and host-driven iterations
    const int grid = kDotBlocks;
    long long chunk = ((c.n + grid - 1) / grid + 63) / 64 * 64;
    int nb = (int)((c.n + chunk - 1) / chunk);
    if (dot)
        k_dot<<<nb, 256, 0, c.st>>>(X, Y, c.n, chunk, c.b->partial, gd);
    else if (p == 1)
        gram_vec_kernel((m + 7) / 8)<<<nb, 256, 0, c.st>>>(X, m, Y, c.ld, c.n, chunk,
                                                            c.b->partial, gd);
    else
        gram_kernel((m + 7) / 8, (p + 7) / 8)<<<nb, 256, 0, c.st>>>(X, m, Y, p, c.ld, c.n,
                                                                     chunk, c.b->partial, gd);
    k_gram_finish<<<m * p, 32, 0, c.st>>>(c.b->partial, nb, m * p, out, gd, p);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

// dots[i] = X_i . y for i < m (device), optionally copied to host
static jci_status dots(Ctx &c, const double *X, int m, const double *y, double *host) {
    jci_status r = gram(c, X, m, y, 1, c.b->dots);
    if (r) return r;
    if (host) {
        JCI_CUDA(cudaMemcpyAsync(host, c.b->dots, m * sizeof(double), cudaMemcpyDeviceToHost,
                                 c.st));
        JCI_CUDA(cudaStreamSynchronize(c.st));
    }
    return JCI_OK;
}

// G[i][j] = V_i . C_j for rows i in [r0, r1) and j <= i (lower triangle):
// one tensor-core product C[0, r1)^T V[i0, i0 + p) per 16 new rows
static jci_status gram_rows(Ctx &c, int r0, int r1, std::vector<double> &G) {
    std::vector<double> h((size_t)kGramRows * kGramCols);
    for (int i0 = r0; i0 < r1; i0 += kGramCols) {
        int p = std::min(kGramCols, r1 - i0), m = i0 + p;
        jci_status r = gram(c, c.b->C, m, c.b->V + i0 * c.ld, p, c.b->dots);
        if (r) return r;
        JCI_CUDA(cudaMemcpyAsync(h.data(), c.b->dots, (size_t)m * p * sizeof(double),
                                 cudaMemcpyDeviceToHost, c.st));
        JCI_CUDA(cudaStreamSynchronize(c.st));
        for (int i = i0; i < i0 + p; i++)
            for (int j = 0; j <= i; j++) G[i * kMaxKry + j] = h[(size_t)j * p + (i - i0)];
    }
    return JCI_OK;
}

// arrow: the device eigenpairs are those of the leading (m-1) block of G
// (the previous step of the same basis), see k_jacobi
static jci_status rayleigh_ritz(Ctx &c, int m, const std::vector<double> &G,
                                std::vector<double> &w, std::vector<double> &Y,
                                bool arrow = false) {
    DavidsonBuffers *b = c.b;
    JCI_CUDA(cudaMemcpyAsync(b->G, G.data(), kMaxKry * kMaxKry * sizeof(double),
                             cudaMemcpyHostToDevice, c.st));
    size_t smem = 2 * (size_t)m * (m + 1) * sizeof(double);
    // the attribute is per device; setting it again is harmless and cheap
    JCI_CUDA(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * kMaxKry * (kMaxKry + 1) * sizeof(double))));
    k_jacobi<<<1, kJacobiThreads, smem, c.st>>>(b->G, m, kMaxKry, b->eval, b->evec, c.d_info,
                                                nullptr, arrow ? 1 : 0);
    int info = 0;
    JCI_CUDA(cudaMemcpyAsync(w.data(), b->eval, m * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaMemcpyAsync(Y.data(), b->evec, kMaxKry * kMaxKry * sizeof(double),
                             cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaMemcpyAsync(&info, c.d_info, sizeof(int), cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaStreamSynchronize(c.st));
    JCI_CUDA(cudaGetLastError());
    return info < 0 ? JCI_ERR_LINALG : JCI_OK;
}

// out = sum_i a[i] X_i + sum_i bb[i] Y_i with host coefficients
static jci_status lincomb(Ctx &c, double *out, const double *X, const double *a, int mx,
                          const double *Yv, const double *bb, int my) {
    DavidsonBuffers *b = c.b;
    std::vector<double> cc(2 * kMaxKry, 0.0);
    for (int i = 0; i < mx; i++) cc[i] = a[i];
    for (int i = 0; i < my; i++) cc[kMaxKry + i] = bb[i];
    JCI_CUDA(cudaMemcpyAsync(b->coef, cc.data(), 2 * kMaxKry * sizeof(double),
                             cudaMemcpyHostToDevice, c.st));
    k_lincomb<<<grid_for(c.n), 256, 0, c.st>>>(out, c.n, c.ld, X, b->coef, mx, Yv,
                                               b->coef + kMaxKry, my, nullptr);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

// V <- V Y^T[:, :k] (and C likewise): Ritz vectors of the first k roots
static jci_status collapse(Ctx &c, int m, int k, const std::vector<double> &Y,
                           bool rotate_c = true) {
    DavidsonBuffers *b = c.b;
    jci_status r;
    for (int pass = 0; pass < (rotate_c ? 2 : 1); pass++) {
        double *src = pass ? b->C : b->V;
        for (int i = 0; i < k; i++)
            if ((r = lincomb(c, b->X + i * c.ld, src, &Y[i * kMaxKry], m, nullptr, nullptr, 0)))
                return r;
        JCI_CUDA(cudaMemcpyAsync(src, b->X, (size_t)k * c.ld * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c.st));
        JCI_CUDA(cudaMemsetAsync(src + k * c.ld, 0, (size_t)(b->cap - k) * c.ld * sizeof(double),
                                 c.st));
    }
    return JCI_OK;
}

// Precision switch of the mixed schedule: collapse the basis to its `keep`
// lowest Ritz vectors from the FP32 phase and recompute only their sigma
// vectors in FP64 (the FP32 sigma vectors of the dropped directions are
// never needed in FP64), then rebuild the subspace matrix.
static jci_status switch_to_fp64(Ctx &c, int &ckdim, int keep, std::vector<double> &G,
                                 std::vector<double> &w, std::vector<double> &Y) {
    jci_status r;
    if (keep < ckdim) {
        if ((r = collapse(c, ckdim, keep, Y, false))) return r;
        ckdim = keep;
    }
    if ((r = sigma_block(c, 0, ckdim, false))) return r;
    if ((r = gram_rows(c, 0, ckdim, G))) return r;
    return rayleigh_ritz(c, ckdim, G, w, Y);
}

// orthonormalise t against V_0..V_{m-1} (npass classical Gram-Schmidt
// passes) and normalise; returns the norm before the final normalisation in
// *nrm.  With prescale, t is first scaled to unit length, so *nrm is the
// fraction of t that lies outside the current space.
static jci_status orthonormalize(Ctx &c, double *t, int m, int npass, double *nrm,
                                 bool prescale = false) {
    DavidsonBuffers *b = c.b;
    jci_status r;
    if (prescale) {
        if ((r = dots(c, t, 1, t, nullptr))) return r;
        k_normalize<<<grid_for(c.n), 256, 0, c.st>>>(t, c.n, b->dots, nullptr);
    }
    for (int p = 0; p < npass && m > 0; p++) {
        if ((r = dots(c, b->V, m, t, nullptr))) return r;
        k_orth_update<<<grid_for(c.n), 256, 0, c.st>>>(t, c.n, c.ld, b->V, b->dots, m, nullptr);
    }
    if ((r = dots(c, t, 1, t, nullptr))) return r;
    double h = 0.0;
    JCI_CUDA(cudaMemcpyAsync(&h, b->dots, sizeof(double), cudaMemcpyDeviceToHost, c.st));
    k_normalize<<<grid_for(c.n), 256, 0, c.st>>>(t, c.n, b->dots, nullptr);
    JCI_CUDA(cudaStreamSynchronize(c.st));
    JCI_CUDA(cudaGetLastError());
    *nrm = sqrt(h);
    return JCI_OK;
}

// Host-side Slater-rule element between two determinants, for the
// prediagonalisation guess (init_diag_H_subspace, pdavidson.c:3963, with
// the generic hmatels of action_util.c:119).
static double host_hmat(const jci_space *s, long long di, long long dj);

static void host_symeig(int n, std::vector<double> a, std::vector<double> &w,
                        std::vector<double> &z);

static jci_status initial_vectors(Ctx &c, const jci_davidson_opts *o) {
    jci_space *s = c.s;
    int kmin = o->krymin;
    long long n = c.n;
    std::vector<double> v0((size_t)kmin * n, 0.0);
    if (o->prediagr == 1) {
        int dim = (int)std::min<long long>(o->refdim, n);
        std::vector<double> h((size_t)dim * dim), w, z;
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < dim; j++) h[i * dim + j] = host_hmat(s, i, j);
        host_symeig(dim, h, w, z);
        for (int i = 0; i < kmin && i < dim; i++)
            for (int j = 0; j < dim; j++) v0[(size_t)i * n + j] = z[(size_t)i * dim + j];
    } else if (o->prediagr == 2) {
        for (int i = 0; i < kmin; i++) v0[(size_t)i * n + i] = 1.0;
    } else {
        if (o->init) {
            memcpy(v0.data(), o->init, sizeof(double) * kmin * n);
        } else {
            jci_status r = jci_read_vectors("ci.restart", kmin, (int)n, v0.data());
            if (r) return r;
        }
    }
    for (int i = 0; i < kmin; i++)
        JCI_CUDA(cudaMemcpyAsync(c.b->V + i * c.ld, &v0[(size_t)i * n], n * sizeof(double),
                                 cudaMemcpyHostToDevice, c.st));
    JCI_CUDA(cudaStreamSynchronize(c.st));
    return JCI_OK;
}

// ---- iterations of the root-sequential schedule ---------------------------
//
// One iteration: residual of the current root, its norm test, the
// preconditioned correction, one classical Gram-Schmidt pass, sigma of the
// new basis vector, the new row of the subspace matrix and the Jacobi
// eigensolve.  host_iteration launches these kernels with sizes known on
// the host and reads the residual norm back; the captured iteration
// (enqueue_iteration) runs the same kernels in the same order with every
// size and decision kept in the device control block, so a batch of graph
// launches needs one host synchronisation instead of five per iteration and
// gives bitwise the same numbers.
//
// event: 0 vector added, 1 residual of root croot below tol (nothing added),
// 2 basis full.

static void print_iteration(const Ctx &c, int citer, int root, double theta, double rn,
                            bool fp32) {
    printf("  iter %4d  root %d  E = %18.12f  ||r|| = %.3e%s\n", citer, root,
           theta + c.s->nucrep + c.s->frzcore, rn, fp32 ? "  (fp32 sigma)" : "");
}

static jci_status host_iteration(Ctx &c, const jci_davidson_opts *o, bool fp32, int croot,
                                 double tol, int &ckdim, int &citer, double &rnorm,
                                 std::vector<double> &G, std::vector<double> &w,
                                 std::vector<double> &Y, int *event) {
    DavidsonBuffers *b = c.b;
    std::vector<double> yc(kMaxKry), ycv(kMaxKry);
    jci_status r;
    double th = w[croot - 1];
    for (int i = 0; i < ckdim; i++) {
        yc[i] = Y[(croot - 1) * kMaxKry + i];
        ycv[i] = -th * yc[i];
    }
    if ((r = lincomb(c, b->r, b->C, yc.data(), ckdim, b->V, ycv.data(), ckdim))) return r;
    double rn2 = 0.0;
    if ((r = dots(c, b->r, 1, b->r, &rn2))) return r;
    rnorm = sqrt(rn2);
    if (o->printlvl > 0) print_iteration(c, citer, croot, th, rnorm, fp32);
    if (rnorm < tol) {
        *event = 1;
        return JCI_OK;
    }
    k_precond<<<grid_for(c.n), 256, 0, c.st>>>(b->r, c.d->hd, th, b->t, c.n, nullptr);
    double nn;
    if ((r = orthonormalize(c, b->t, ckdim, 1, &nn))) return r;
    JCI_CUDA(cudaMemcpyAsync(b->V + ckdim * c.ld, b->t, c.n * sizeof(double),
                             cudaMemcpyDeviceToDevice, c.st));
    if ((r = sigma_block(c, ckdim, 1, fp32))) return r;
    ckdim++;
    if ((r = gram_rows(c, ckdim - 1, ckdim, G))) return r;
    if ((r = rayleigh_ritz(c, ckdim, G, w, Y, true))) return r;
    citer++;
    *event = ckdim >= o->krymax ? 2 : 0;
    return JCI_OK;
}

static jci_status enqueue_iteration(Ctx &c, bool fp32, int kmax) {
    DavidsonBuffers *b = c.b;
    DavCtl *ctl = b->ctl;
    const int *stop = &ctl->stop;
    const unsigned g = grid_for(c.n);
    GramDev one, basis, with_new;
    one.stop = basis.stop = with_new.stop = stop;
    basis.mdev = with_new.mdev = &ctl->ckdim;
    with_new.madd = 1;
    jci_status r;
    k_it_begin<<<1, 64, 0, c.st>>>(ctl, b->eval, b->evec, b->coef);
    k_lincomb<<<g, 256, 0, c.st>>>(b->r, c.n, c.ld, b->C, b->coef, 0, b->V, b->coef + kMaxKry,
                                   0, ctl);
    if ((r = gram(c, b->r, 1, b->r, 1, b->dots, one))) return r;
    k_it_check<<<1, 1, 0, c.st>>>(ctl, b->dots, b->hist);
    k_precond<<<g, 256, 0, c.st>>>(b->r, c.d->hd, 0.0, b->t, c.n, ctl);
    // the row counts below come from the control block; kmax bounds them
    if ((r = gram(c, b->V, kmax, b->t, 1, b->dots, basis))) return r;
    k_orth_update<<<g, 256, 0, c.st>>>(b->t, c.n, c.ld, b->V, b->dots, 0, ctl);
    if ((r = gram(c, b->t, 1, b->t, 1, b->dots, one))) return r;
    k_normalize<<<g, 256, 0, c.st>>>(b->t, c.n, b->dots, stop);
    k_it_store<<<g, 256, 0, c.st>>>(b->V, c.ld, 0, b->t, c.n, ctl);
    if (fp32) {
        k_d2f<<<g, 256, 0, c.st>>>(b->t, b->v32, c.n, c.ld, c.ld, 1, stop);
        if ((r = device_sigma(c.s, 1, b->v32, b->s32, c.ld, JCI_FP32, c.st))) return r;
        k_f2d<<<g, 256, 0, c.st>>>(b->s32, b->cnew, c.n, c.ld, c.ld, 1, stop);
    } else {
        if ((r = device_sigma(c.s, 1, b->t, b->cnew, c.ld, JCI_FP64, c.st))) return r;
    }
    k_it_store<<<g, 256, 0, c.st>>>(b->C, c.ld, 0, b->cnew, c.n, ctl);
    if ((r = gram(c, b->C, kmax, b->t, 1, b->dots, with_new))) return r;
    k_it_append<<<1, 64, 0, c.st>>>(ctl, b->dots, b->G);
    k_jacobi<<<1, kJacobiThreads, 2 * (size_t)kmax * (kmax + 1) * sizeof(double), c.st>>>(
        b->G, 0, kMaxKry, b->eval, b->evec, b->info, ctl, 1);
    k_it_end<<<1, 1, 0, c.st>>>(ctl, b->info, kmax);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

// Capture (once per precision, basis size and sigma plan) the iteration as
// a CUDA graph.  The sigma kernels see the control block's stop flag.
static jci_status ensure_graph(Ctx &c, bool fp32, int kmax) {
    DavidsonBuffers *b = c.b;
    const int p = fp32 ? 1 : 0;
    int plan[4] = {0, 0, 0, 0};
    if (c.d->fci) {
        float ms = 0.f;
        fci_tuning(c.s, fp32 ? JCI_FP32 : JCI_FP64, &plan[0], &plan[1], &plan[2], &plan[3], &ms);
    }
    if (b->gexec[p] && b->gkmax[p] == kmax && memcmp(plan, b->gplan[p], sizeof plan) == 0)
        return JCI_OK;
    if (b->gexec[p]) {
        cudaGraphExecDestroy(b->gexec[p]);
        b->gexec[p] = nullptr;
    }
    JCI_CUDA(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * kMaxKry * (kMaxKry + 1) * sizeof(double))));
    cudaGraph_t graph = nullptr;
    JCI_CUDA(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeRelaxed));
    c.d->sigma_skip = &b->ctl->stop;
    jci_status r = enqueue_iteration(c, fp32, kmax);
    c.d->sigma_skip = nullptr;
    cudaError_t e = cudaStreamEndCapture(c.st, &graph);
    if (r == JCI_OK && e != cudaSuccess) r = cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    if (r == JCI_OK) {
        e = cudaGraphInstantiate(&b->gexec[p], graph, 0);
        if (e != cudaSuccess) {
            b->gexec[p] = nullptr;
            r = cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
        }
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (r) return r;
    b->gkmax[p] = kmax;
    memcpy(b->gplan[p], plan, sizeof plan);
    return JCI_OK;
}

// Launch the captured iteration kmax - ckdim times (the last launch fills
// the basis at the latest), then read the control block, the history and
// the subspace state back in one synchronisation.
static jci_status graph_iterations(Ctx &c, const jci_davidson_opts *o, bool fp32, int croot,
                                   double tol, int &ckdim, int &citer, double &rnorm,
                                   std::vector<double> &G, std::vector<double> &w,
                                   std::vector<double> &Y, int *event) {
    DavidsonBuffers *b = c.b;
    const int kmax = o->krymax, p = fp32 ? 1 : 0;
    jci_status r = ensure_graph(c, fp32, kmax);
    if (r) return r;
    DavCtl h{};
    h.ckdim = ckdim;
    h.croot = croot - 1;
    h.tol = tol;
    JCI_CUDA(cudaMemcpyAsync(b->ctl, &h, sizeof h, cudaMemcpyHostToDevice, c.st));
    for (int k = ckdim; k < kmax; k++) JCI_CUDA(cudaGraphLaunch(b->gexec[p], c.st));
    std::vector<DavHist> hist(kHist);
    JCI_CUDA(cudaMemcpyAsync(&h, b->ctl, sizeof h, cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaMemcpyAsync(hist.data(), b->hist, kHist * sizeof(DavHist),
                             cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaMemcpyAsync(w.data(), b->eval, kMaxKry * sizeof(double), cudaMemcpyDeviceToHost,
                             c.st));
    JCI_CUDA(cudaMemcpyAsync(Y.data(), b->evec, kMaxKry * kMaxKry * sizeof(double),
                             cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaMemcpyAsync(G.data(), b->G, kMaxKry * kMaxKry * sizeof(double),
                             cudaMemcpyDeviceToHost, c.st));
    JCI_CUDA(cudaStreamSynchronize(c.st));
    if ((r = fci_wait_status(c.s))) return r;
    const int nh = std::min(h.nhist, kHist);
    for (int i = 0; i < nh; i++) {
        rnorm = hist[i].rnorm;
        if (o->printlvl > 0)
            print_iteration(c, citer + i, hist[i].root + 1, hist[i].theta, hist[i].rnorm, fp32);
    }
    ckdim = h.ckdim;
    citer += h.iters;
    c.sigma_calls += h.iters;
    c.sigma_vecs += h.iters;
    if (fp32) c.fp32_vecs += h.iters;
    c.sigma_ms += h.iters * c.ms_per_vec[p];
    if (h.stop == 3) return JCI_ERR_LINALG;
    *event = h.stop == 1 ? 1 : 2;
    return JCI_OK;
}

// Residual norm of root croot in the current subspace, on the host path:
// r = sum_i y_i (c_i - theta v_i).
static jci_status residual_norm(Ctx &c, int ckdim, int croot, const std::vector<double> &w,
                                const std::vector<double> &Y, double *rn) {
    DavidsonBuffers *b = c.b;
    std::vector<double> yc(kMaxKry), ycv(kMaxKry);
    const double th = w[croot - 1];
    for (int i = 0; i < ckdim; i++) {
        yc[i] = Y[(croot - 1) * kMaxKry + i];
        ycv[i] = -th * yc[i];
    }
    jci_status r = lincomb(c, b->r, b->C, yc.data(), ckdim, b->V, ycv.data(), ckdim);
    if (r) return r;
    double rn2 = 0.0;
    if ((r = dots(c, b->r, 1, b->r, &rn2))) return r;
    *rn = sqrt(rn2);
    return JCI_OK;
}

// Anchor of the mixed refinement phase: collapse the basis to the kmin
// lowest Ritz vectors (sigma vectors rotated with them), recompute the
// sigma of basis vectors [r0, r1) -- the Ritz vectors of the roots being
// refined -- in FP64, and rebuild the subspace matrix and the Ritz pairs.
static jci_status anchor(Ctx &c, int &ckdim, int kmin, int r0, int r1, std::vector<double> &G,
                         std::vector<double> &w, std::vector<double> &Y) {
    jci_status r;
    if ((r = collapse(c, ckdim, kmin, Y, true))) return r;
    ckdim = kmin;
    if ((r = sigma_block(c, r0, r1 - r0, false))) return r;
    if ((r = gram_rows(c, 0, ckdim, G))) return r;
    return rayleigh_ritz(c, ckdim, G, w, Y);
}

// Residual reduction asked of the FP32-sigma corrections between two
// anchors of the mixed refinement phase.  A correction's FP32 sigma carries
// an error of about 1e-6 ||H|| per unit vector, but it enters the current
// root's residual only through that correction's coefficient in the Ritz
// vector, which is of the order of the residual at the last anchor divided
// by the gap to the next root; two decades per anchor stay well above that
// floor.
constexpr double kRefineStep = 1e-2;

static jci_status run_sequential(Ctx &c, const jci_davidson_opts *o, bool mixed,
                                 std::vector<double> &w, std::vector<double> &Y, int &ckdim,
                                 int &citer, int &converged, double &rnorm) {
    std::vector<double> G(kMaxKry * kMaxKry, 0.0);
    int kmin = o->krymin, kmax = o->krymax, nroots = o->nroots;
    bool fp32 = mixed;
    // The reference recomputes every sigma vector after a collapse
    // (pdavidson.c:39 loop); the mixed schedule rotates them with the Ritz
    // coefficients instead (the same vectors in exact arithmetic).
    const bool recompute = !mixed;
    // Mixed: phase 1 takes every root, one after the other, below
    // switch_tol with FP32 sigma.  The switch collapses to the krymin lowest
    // Ritz vectors and recomputes their sigma in FP64.  Phase 2 refines the
    // roots from the first to restol: new correction vectors keep FP32
    // sigma, and every stop of the graph-driven iterations (the current
    // root's residual below its step target, or a full basis) anchors that
    // root -- collapse, FP64 sigma of its Ritz vector, new subspace matrix
    // -- so its residual is measured again with FP64 sigma.  A root counts
    // as converged only on a residual taken right after its anchor; at the
    // end every root's Ritz vector gets an FP64 sigma and every residual is
    // checked again.
    double tol = mixed ? o->switch_tol : o->restol;
    bool refine = false;
    int croot = 1, cflag = 0;
    bool have_sigma = false;
    ckdim = kmin;
    citer = 1;
    jci_status r;
    // step target of root k in phase 2 from its residual rn
    auto target = [&](double rn) { return std::max(o->restol, rn * kRefineStep); };
    while (citer < o->maxiter && croot <= nroots) {
        if (recompute || !have_sigma) {
            if ((r = sigma_block(c, 0, ckdim, fp32))) return r;
            have_sigma = true;
        }
        if ((r = gram_rows(c, 0, ckdim, G))) return r;
        if ((r = rayleigh_ritz(c, ckdim, G, w, Y))) return r;
        for (;;) {
            int event = 2;
            if (ckdim < kmax) {
                r = o->host_loop
                        ? host_iteration(c, o, fp32, croot, tol, ckdim, citer, rnorm, G, w, Y,
                                         &event)
                        : graph_iterations(c, o, fp32, croot, tol, ckdim, citer, rnorm, G, w,
                                           Y, &event);
                if (r) return r;
            }
            if (event == 0) continue;
            if (refine) {
                if ((r = anchor(c, ckdim, kmin, croot - 1, croot, G, w, Y))) return r;
                double rn = 0.0;
                if ((r = residual_norm(c, ckdim, croot, w, Y, &rn))) return r;
                rnorm = rn;
                if (rn < o->restol) {
                    if (croot < nroots) {
                        croot++;
                        if ((r = residual_norm(c, ckdim, croot, w, Y, &rn))) return r;
                    } else {
                        // every root: FP64 sigma of its Ritz vector, residual again
                        if ((r = anchor(c, ckdim, kmin, 0, nroots, G, w, Y))) return r;
                        int bad = 0;
                        for (int k = 1; k <= nroots && !bad; k++) {
                            if ((r = residual_norm(c, ckdim, k, w, Y, &rn))) return r;
                            rnorm = std::max(rnorm, rn);
                            if (rn >= o->restol) bad = k;
                        }
                        if (!bad) {
                            // leave the Ritz vectors of this last eigensolve in
                            // the basis, as a collapse does
                            if ((r = collapse(c, ckdim, kmin, Y, true))) return r;
                            ckdim = kmin;
                            cflag = 2;
                            break;
                        }
                        croot = bad;
                    }
                }
                tol = target(rn);
                if (citer >= o->maxiter) break;
                continue;
            }
            if (event == 2) {
                cflag = 0;
                break;
            }
            cflag = croot < nroots ? 1 : 2;
            if (cflag == 2 && fp32) {
                refine = true;
                croot = 1;
                cflag = 0;
                if ((r = switch_to_fp64(c, ckdim, kmin, G, w, Y))) return r;
                double rn = 0.0;
                if ((r = residual_norm(c, ckdim, croot, w, Y, &rn))) return r;
                tol = target(rn);
                continue;
            }
            if (cflag == 1) croot++;
            break;
        }
        if (cflag == 2 && refine) break;
        if (refine) break;  // maxiter reached inside the refinement phase
        if ((r = collapse(c, ckdim, kmin, Y, !recompute))) return r;
        ckdim = kmin;
        if (cflag == 2) break;
    }
    converged = cflag == 2;
    return JCI_OK;
}

static jci_status run_block(Ctx &c, const jci_davidson_opts *o, bool mixed,
                            std::vector<double> &w, std::vector<double> &Y, int &ckdim,
                            int &citer, int &converged, double &rnorm) {
    DavidsonBuffers *b = c.b;
    std::vector<double> G(kMaxKry * kMaxKry, 0.0), yc(kMaxKry), ycv(kMaxKry);
    int kmin = o->krymin, kmax = o->krymax, nroots = o->nroots;
    bool fp32 = mixed;
    ckdim = kmin;
    citer = 1;
    jci_status r;
    if ((r = sigma_block(c, 0, ckdim, fp32))) return r;
    if ((r = gram_rows(c, 0, ckdim, G))) return r;
    if ((r = rayleigh_ritz(c, ckdim, G, w, Y))) return r;
    converged = 0;
    while (citer < o->maxiter) {
        // residuals of all roots
        std::vector<double> rn(nroots);
        double rmax = 0.0;
        for (int k = 0; k < nroots; k++) {
            double th = w[k];
            for (int i = 0; i < ckdim; i++) {
                yc[i] = Y[k * kMaxKry + i];
                ycv[i] = -th * yc[i];
            }
            if ((r = lincomb(c, b->r, b->C, yc.data(), ckdim, b->V, ycv.data(), ckdim))) return r;
            double rn2 = 0.0;
            if ((r = dots(c, b->r, 1, b->r, &rn2))) return r;
            rn[k] = sqrt(rn2);
            rmax = std::max(rmax, rn[k]);
        }
        rnorm = rmax;
        if (o->printlvl > 0) {
            printf("  iter %4d  dim %2d ", citer, ckdim);
            for (int k = 0; k < nroots; k++)
                printf(" E%d = %.12f (%.2e)", k + 1, w[k] + c.s->nucrep + c.s->frzcore, rn[k]);
            printf("%s\n", fp32 ? "  fp32" : "");
        }
        if (fp32 && rmax < o->switch_tol) {
            fp32 = false;
            if ((r = switch_to_fp64(c, ckdim, std::max(kmin, nroots), G, w, Y))) return r;
            continue;
        }
        if (rmax < o->restol) {
            converged = 1;
            break;
        }
        int nnew = 0;
        for (int k = 0; k < nroots; k++) if (rn[k] >= o->restol) nnew++;
        if (ckdim + nnew > kmax) {
            int keep = std::max(kmin, nroots);
            if ((r = collapse(c, ckdim, keep, Y))) return r;
            ckdim = keep;
            if ((r = gram_rows(c, 0, ckdim, G))) return r;
            if ((r = rayleigh_ritz(c, ckdim, G, w, Y))) return r;
            continue;
        }
        int added = 0;
        for (int k = 0; k < nroots; k++) {
            if (rn[k] < o->restol) continue;
            double th = w[k];
            for (int i = 0; i < ckdim; i++) {
                yc[i] = Y[k * kMaxKry + i];
                ycv[i] = -th * yc[i];
            }
            if ((r = lincomb(c, b->r, b->C, yc.data(), ckdim, b->V, ycv.data(), ckdim))) return r;
            k_precond<<<grid_for(c.n), 256, 0, c.st>>>(b->r, c.d->hd, th, b->t, c.n, nullptr);
            double nn;
            if ((r = orthonormalize(c, b->t, ckdim + added, 2, &nn, true))) return r;
            if (!(nn > 1e-8)) continue;  // correction (numerically) inside the space
            JCI_CUDA(cudaMemcpyAsync(b->V + (ckdim + added) * c.ld, b->t, c.n * sizeof(double),
                                     cudaMemcpyDeviceToDevice, c.st));
            added++;
        }
        if (added == 0) break;
        if ((r = sigma_block(c, ckdim, added, fp32))) return r;
        ckdim += added;
        if ((r = gram_rows(c, ckdim - added, ckdim, G))) return r;
        if ((r = rayleigh_ritz(c, ckdim, G, w, Y))) return r;
        citer += added;
    }
    if ((r = collapse(c, ckdim, std::max(kmin, nroots), Y))) return r;
    ckdim = std::max(kmin, nroots);
    return JCI_OK;
}

jci_status davidson(jci_space *s, const jci_davidson_opts *o, double *energies, double *civec,
                    jci_davidson_stats *stats) {
    auto t0 = std::chrono::steady_clock::now();
    if (!s->have_ints) return JCI_ERR_STATE;
    if (o->krymin < o->nroots || o->krymax < o->krymin || o->krymax > kMaxKry ||
        o->nroots < 1 || o->krymax > s->ndets || o->maxiter < 1)
        return JCI_ERR_ARG;
    Ctx c;
    c.s = s;
    c.d = s->dev;
    c.st = c.d->stream;
    c.n = s->ndets;
    JCI_CUDA(cudaSetDevice(c.d->device));
    bool mixed = o->precision == JCI_MIXED;
    int maxnew = std::max(o->krymin, o->nroots);
    jci_status r = ensure_buffers(c, o->krymax, mixed, maxnew);
    if (r) return r;
    c.d_info = c.b->info;
    std::vector<double> w(kMaxKry, 0.0), Y(kMaxKry * kMaxKry, 0.0);
    int ckdim = 0, citer = 0, conv = 0;
    double rnorm = 0.0;
    r = initial_vectors(c, o);
    if (!r) {
        if (o->block)
            r = run_block(c, o, mixed, w, Y, ckdim, citer, conv, rnorm);
        else
            r = run_sequential(c, o, mixed, w, Y, ckdim, citer, conv, rnorm);
    }
    if (r) return r;
    // a product kernel that gave up a bounded wait left its sigma incomplete
    if ((r = fci_wait_status(s))) return r;
    double core = s->nucrep + s->frzcore;
    for (int k = 0; k < o->nroots; k++) energies[k] = w[k] + core;
    std::vector<double> host;
    if (civec || o->write_files) {
        host.resize((size_t)std::max(o->krymin, o->nroots) * c.n);
        for (int k = 0; k < std::max(o->krymin, o->nroots); k++)
            JCI_CUDA(cudaMemcpyAsync(&host[(size_t)k * c.n], c.b->V + k * c.ld,
                                     c.n * sizeof(double), cudaMemcpyDeviceToHost, c.st));
        JCI_CUDA(cudaStreamSynchronize(c.st));
        if (civec) memcpy(civec, host.data(), sizeof(double) * o->nroots * c.n);
    }
    if (o->write_files) {
        // pdavidson.c:343-347
        if ((r = jci_write_vectors("civec", o->nroots, (int)c.n, host.data()))) return r;
        if (!conv) {
            if ((r = jci_write_vectors("ci.restart", o->krymin, (int)c.n, host.data()))) return r;
            std::vector<double> hv((size_t)o->nroots * c.n);
            for (int k = 0; k < o->nroots; k++)
                JCI_CUDA(cudaMemcpy(&hv[(size_t)k * c.n], c.b->C + k * c.ld,
                                    c.n * sizeof(double), cudaMemcpyDeviceToHost));
            if ((r = jci_write_vectors("hvvec", o->nroots, (int)c.n, hv.data()))) return r;
        }
    }
    if (stats) {
        stats->iterations = citer;
        stats->sigma_calls = c.sigma_calls;
        stats->sigma_vectors = c.sigma_vecs;
        stats->sigma_seconds = c.sigma_ms * 1e-3;
        stats->total_seconds =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        stats->converged = conv;
        stats->rnorm = rnorm;
        stats->fp32_sigma_vectors = c.fp32_vecs;
    }
    return conv ? JCI_OK : JCI_ERR_NOCONV;
}

// First k basis vectors left by the last solve on this handle (after the
// final collapse these are the Ritz vectors of the lowest k roots).
jci_status davidson_vectors(jci_space *s, int k, double *out) {
    DeviceState *d = s->dev;
    if (!d || !d->dav || k > d->dav->cap) return JCI_ERR_STATE;
    DavidsonBuffers *b = d->dav;
    for (int i = 0; i < k; i++)
        JCI_CUDA(cudaMemcpyAsync(out + (size_t)i * s->ndets, b->V + i * b->ld,
                                 s->ndets * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
    JCI_CUDA(cudaStreamSynchronize(d->stream));
    return JCI_OK;
}

// ---- host helpers --------------------------------------------------------

static inline double h1(const jci_space *s, int i, int j) {
    return s->m1[pair_index(i, j)];
}
static inline double h2(const jci_space *s, int i, int j, int k, int l) {
    return s->m2[eri_index(pair_index(i, j), pair_index(k, l))];
}

static int phase(const int *o, int ne, int io, int fo) {
    int lo = std::min(io, fo), hi = std::max(io, fo), c = 0;
    for (int i = 0; i < ne; i++) c += (o[i] > lo && o[i] < hi);
    return (c & 1) ? -1 : 1;
}

static double host_hmat(const jci_space *s, long long di, long long dj) {
    int k, pi, qi, pj, qj;
    det_strings(s, di, &k, &pi, &qi);
    det_strings(s, dj, &k, &pj, &qj);
    int na = s->sp[0].nelec, nb = s->sp[1].nelec;
    const int *ai = &s->sp[0].istr[(size_t)pi * na], *aj = &s->sp[0].istr[(size_t)pj * na];
    const int *bi = &s->sp[1].istr[(size_t)qi * nb], *bj = &s->sp[1].istr[(size_t)qj * nb];
    auto diff = [](const int *x, const int *y, int n, int *out) {
        int c = 0;
        for (int i = 0; i < n; i++) {
            bool f = false;
            for (int j = 0; j < n; j++) f |= (x[i] == y[j]);
            if (!f) out[c++] = x[i];
        }
        return c;
    };
    int ax[kMaxElec], af[kMaxElec], bx[kMaxElec], bf[kMaxElec];
    int nax = diff(ai, aj, na, ax), nbx = diff(bi, bj, nb, bx);
    diff(aj, ai, na, af);
    diff(bj, bi, nb, bf);
    if (nax + nbx > 2) return 0.0;
    auto one = [&](const int *o1, int n1, int io, int fo, const int *o2, int n2) {
        double v = h1(s, io, fo);
        for (int i = 0; i < n1; i++)
            if (o1[i] != io) v += h2(s, o1[i], o1[i], io, fo) - h2(s, o1[i], io, o1[i], fo);
        for (int i = 0; i < n2; i++) v += h2(s, o2[i], o2[i], io, fo);
        return phase(o1, n1, io, fo) * v;
    };
    if (nax + nbx == 0) {
        double v = 0.0;
        for (int i = 0; i < na; i++) {
            v += h1(s, ai[i], ai[i]);
            for (int j = 0; j < i; j++)
                v += h2(s, ai[i], ai[i], ai[j], ai[j]) - h2(s, ai[i], ai[j], ai[i], ai[j]);
        }
        for (int i = 0; i < nb; i++) {
            v += h1(s, bi[i], bi[i]);
            for (int j = 0; j < i; j++)
                v += h2(s, bi[i], bi[i], bi[j], bi[j]) - h2(s, bi[i], bi[j], bi[i], bi[j]);
        }
        for (int i = 0; i < na; i++)
            for (int j = 0; j < nb; j++) v += h2(s, ai[i], ai[i], bi[j], bi[j]);
        return v;
    }
    if (nax == 1 && nbx == 0) return one(ai, na, ax[0], af[0], bi, nb);
    if (nax == 0 && nbx == 1) return one(bi, nb, bx[0], bf[0], ai, na);
    if (nax == 1 && nbx == 1)
        return phase(ai, na, ax[0], af[0]) * phase(bi, nb, bx[0], bf[0]) *
               h2(s, ax[0], af[0], bx[0], bf[0]);
    const int *o = nax == 2 ? ai : bi;
    int n = nax == 2 ? na : nb;
    int *x = nax == 2 ? ax : bx, *f = nax == 2 ? af : bf;
    // io = (higher, lower), fo ascending; phase of the first replacement in
    // the string times that of the second in the intermediate string
    int t1[kMaxElec], m = 0;
    for (int i = 0; i < n; i++)
        if (o[i] != x[1]) t1[m++] = o[i];
    int kk = m;
    while (kk > 0 && t1[kk - 1] > f[0]) {
        t1[kk] = t1[kk - 1];
        kk--;
    }
    t1[kk] = f[0];
    int p = phase(o, n, x[1], f[0]) * phase(t1, n, x[0], f[1]);
    return p * (h2(s, x[1], f[0], x[0], f[1]) - h2(s, x[1], f[1], x[0], f[0]));
}

static void host_symeig(int n, std::vector<double> a, std::vector<double> &w,
                        std::vector<double> &z) {
    std::vector<double> v((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) v[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) off += a[p * n + q] * a[p * n + q];
        if (off < 1e-30) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = a[p * n + q];
                if (fabs(apq) < 1e-300) continue;
                double th = (a[q * n + q] - a[p * n + p]) / (2 * apq);
                double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                double cc = 1.0 / sqrt(t * t + 1.0), ss = t * cc;
                for (int k = 0; k < n; k++) {
                    double akp = a[k * n + p], akq = a[k * n + q];
                    a[k * n + p] = cc * akp - ss * akq;
                    a[k * n + q] = ss * akp + cc * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = a[p * n + k], aqk = a[q * n + k];
                    a[p * n + k] = cc * apk - ss * aqk;
                    a[q * n + k] = ss * apk + cc * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double vkp = v[k * n + p], vkq = v[k * n + q];
                    v[k * n + p] = cc * vkp - ss * vkq;
                    v[k * n + q] = ss * vkp + cc * vkq;
                }
            }
    }
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(),
                     [&](int x, int y) { return a[x * n + x] < a[y * n + y]; });
    w.assign(n, 0.0);
    z.assign((size_t)n * n, 0.0);
    for (int k = 0; k < n; k++) {
        w[k] = a[ord[k] * n + ord[k]];
        for (int i = 0; i < n; i++) z[(size_t)k * n + i] = v[(size_t)i * n + ord[k]];
    }
}

}  // namespace jci
