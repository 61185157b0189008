// jci_dyson.cu -- Dyson orbitals between an (N+1)-electron and an
// N-electron CI wavefunction (the reference's pdycicalc program:
// run_pdycicalc.c:376-414 with compute_dyson_orbital_a / _b and
// generate_strcontlist, dysoncomp.c:103-491).
//
// For every determinant I = (p, q) of the (N+1) space and every electron of
// the spin whose count differs between the two wavefunctions (beta when
// N+1 is even, alpha when odd), the electron in orbital o is removed; when
// the resulting string exists in the N space and the (p', q') group pair is
// allowed there, the determinant J of the N space gives
//     d_jk[o] += c0_j(I) c1_k(J)
// (no phase factor: the reference accumulates plain products), and every
// Dyson orbital is scaled by sqrt(N+1).
//
// Layout: the removal targets are tabulated per string of the compared
// spin, rem[x][o] = index of string x without orbital o+1 in the N space,
// or -1.  One CTA takes a contiguous range of (N+1) determinants; for each
// orbital its threads accumulate their determinants' products in registers,
// the CTA reduces them in a fixed order into per-CTA partials, and a second
// kernel sums the partials in CTA order, so the result is bitwise
// reproducible.  The work is bounded by the (N+1) vectors (each read once
// per orbital, from L2 for the sizes of interest) and a gather of the N
// vectors.
#include <cmath>
#include <cstring>
#include <vector>

#include "jci_device.cuh"

namespace jci {

constexpr int kDysMaxPairs = 25;  // 5 x 5 states (the &dysonorbital limit)
constexpr int kDysThreads = 256;
constexpr int kDysBlocks = 148 * 4;

__device__ __forceinline__ long long dys_det_index(const SpaceView &v, int p, int q) {
    int gp = v.a.grp[p], gq = v.b.grp[q];
    int k = v.pairidx[gp * v.qegrps + gq];
    if (k < 0) return -1;
    return v.pqoff[k] + (long long)(p - v.a.gstart[gp]) * v.b.gnstr[gq] + (q - v.b.gstart[gq]);
}

// partial[(blk * norb + o) * npr + j*nst1 + k] over this CTA's determinants
__global__ void __launch_bounds__(kDysThreads)
    k_dyson(SpaceView v0, SpaceView v1, int sp, const int *__restrict__ rem, int norb,
            const double *__restrict__ V0, int nst0, const double *__restrict__ V1, int nst1,
            long long chunk, double *__restrict__ partial) {
    __shared__ double red[kDysThreads / 32][kDysMaxPairs];
    const int npr = nst0 * nst1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long lo = (long long)blockIdx.x * chunk, hi = min(v0.ndets, lo + chunk);
    for (int o = 0; o < norb; o++) {
        double acc[kDysMaxPairs];
#pragma unroll
        for (int t = 0; t < kDysMaxPairs; t++) acc[t] = 0.0;
        for (long long i = lo + tid; i < hi; i += kDysThreads) {
            int k = 0;
            while (k + 1 < v0.npq && v0.pqoff[k + 1] <= i) k++;
            int pg = v0.pqg[2 * k], qg = v0.pqg[2 * k + 1];
            long long r = i - v0.pqoff[k];
            int nq = v0.b.gnstr[qg];
            int p = v0.a.gstart[pg] + (int)(r / nq), q = v0.b.gstart[qg] + (int)(r % nq);
            int y = rem[(long long)(sp ? q : p) * norb + o];
            if (y < 0) continue;
            long long J = sp ? dys_det_index(v1, p, y) : dys_det_index(v1, y, q);
            if (J < 0) continue;
#pragma unroll
            for (int t = 0; t < kDysMaxPairs; t++) {
                if (t >= npr) break;
                acc[t] += V0[(long long)(t / nst1) * v0.ndets + i] *
                          V1[(long long)(t % nst1) * v1.ndets + J];
            }
        }
#pragma unroll
        for (int t = 0; t < kDysMaxPairs; t++) {
            if (t >= npr) break;
            double s = acc[t];
            for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
            if (lane == 0) red[warp][t] = s;
        }
        __syncthreads();
        if (tid < npr) {
            double s = 0.0;
            for (int w = 0; w < kDysThreads / 32; w++) s += red[w][tid];
            partial[((long long)blockIdx.x * norb + o) * npr + tid] = s;
        }
        __syncthreads();
    }
}

// out[t * norbs + o] = scale * sum_blk partial[(blk*norb + o)*npr + t]
__global__ void k_dyson_finish(const double *__restrict__ partial, int nblk, int norb, int npr,
                               int norbs, double scale, double *out) {
    const int e = blockIdx.x;  // o * npr + t
    const int o = e / npr, t = e % npr;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblk; b += 32) s += partial[((long long)b * norb + o) * npr + t];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) out[(long long)t * norbs + o] = scale * s;
}

}  // namespace jci

using namespace jci;

namespace {

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { cudaFree(p); }
};

}  // namespace

extern "C" jci_status jci_dyson(jci_space *s0, jci_space *s1, const double *v0, int nstates0,
                                const double *v1, int nstates1, const int *states0, int nst0,
                                const int *states1, int nst1, double *dyorb) {
    if (!s0 || !s1 || !v0 || !v1 || !states0 || !states1 || !dyorb) return JCI_ERR_ARG;
    if (nst0 < 1 || nst1 < 1 || nst0 * nst1 > kDysMaxPairs) return JCI_ERR_ARG;
    for (int j = 0; j < nst0; j++)
        if (states0[j] < 1 || states0[j] > nstates0) return JCI_ERR_ARG;
    for (int k = 0; k < nst1; k++)
        if (states1[k] < 1 || states1[k] > nstates1) return JCI_ERR_ARG;
    // check_wavefunction_input (run_pdycicalc.c:458-489)
    if (s1->electrons != s0->electrons - 1 || s1->orbitals != s0->orbitals ||
        s1->nfrzc != s0->nfrzc || s1->ndocc != s0->ndocc || s1->nactv != s0->nactv ||
        s1->nfrzv != s0->nfrzv)
        return JCI_ERR_ARG;
    const int sp = s0->electrons % 2 == 0 ? 1 : 0;  // the spin that loses an electron
    const int xs = 1 - sp;
    // the other spin's strings are shared (run_pdycicalc.c:362-375)
    if (s0->sp[xs].nstr != s1->sp[xs].nstr || s0->sp[xs].istr != s1->sp[xs].istr ||
        s0->sp[sp].nelec != s1->sp[sp].nelec + 1)
        return JCI_ERR_SPACE;
    const int norb = s0->ci_orbs, ne = s0->sp[sp].nelec;
    const int nx = s0->sp[sp].nstr;
    std::vector<int> rem((size_t)nx * norb, -1), r(ne > 0 ? ne : 1);
    for (int x = 0; x < nx; x++) {
        const int *o = &s0->sp[sp].istr[(size_t)x * ne];
        for (int e = 0; e < ne; e++) {
            int n = 0;
            for (int f = 0; f < ne; f++)
                if (f != e) r[n++] = o[f];
            rem[(size_t)x * norb + o[e] - 1] = string_index(s1, sp, r.data());
        }
    }
    jci_status st;
    for (jci_space *s : {s0, s1})
        if (!s->dev && (st = device_init(s))) return st;
    DeviceState *d0 = s0->dev;
    JCI_CUDA(cudaSetDevice(d0->device));
    cudaStream_t stm = d0->stream;
    JCI_CUDA(cudaStreamSynchronize(s1->dev->stream));  // s1's tables are uploaded
    const int npr = nst0 * nst1;
    const long long n0 = s0->ndets, n1 = s1->ndets;
    long long chunk = (n0 + kDysBlocks - 1) / kDysBlocks;
    chunk = (chunk + kDysThreads - 1) / kDysThreads * kDysThreads;
    const int nblk = (int)((n0 + chunk - 1) / chunk);
    DevBuf dv0, dv1, drem, dpart, dout;
    JCI_CUDA(cudaMalloc(&dv0.p, sizeof(double) * n0 * nst0));
    JCI_CUDA(cudaMalloc(&dv1.p, sizeof(double) * n1 * nst1));
    JCI_CUDA(cudaMalloc(&drem.p, sizeof(int) * rem.size()));
    JCI_CUDA(cudaMalloc(&dpart.p, sizeof(double) * (size_t)nblk * norb * npr));
    const int norbs = s0->orbitals;
    JCI_CUDA(cudaMalloc(&dout.p, sizeof(double) * (size_t)npr * norbs));
    for (int j = 0; j < nst0; j++)
        JCI_CUDA(cudaMemcpyAsync((double *)dv0.p + j * n0, v0 + (size_t)(states0[j] - 1) * n0,
                                 sizeof(double) * n0, cudaMemcpyHostToDevice, stm));
    for (int k = 0; k < nst1; k++)
        JCI_CUDA(cudaMemcpyAsync((double *)dv1.p + k * n1, v1 + (size_t)(states1[k] - 1) * n1,
                                 sizeof(double) * n1, cudaMemcpyHostToDevice, stm));
    JCI_CUDA(cudaMemcpyAsync(drem.p, rem.data(), sizeof(int) * rem.size(),
                             cudaMemcpyHostToDevice, stm));
    JCI_CUDA(cudaMemsetAsync(dout.p, 0, sizeof(double) * (size_t)npr * norbs, stm));
    SpaceView w0 = make_view(s0->dev), w1 = make_view(s1->dev);
    w0.ndets = n0;
    w1.ndets = n1;
    k_dyson<<<nblk, kDysThreads, 0, stm>>>(w0, w1, sp, (const int *)drem.p, norb,
                                           (const double *)dv0.p, nst0, (const double *)dv1.p,
                                           nst1, chunk, (double *)dpart.p);
    k_dyson_finish<<<norb * npr, 32, 0, stm>>>((const double *)dpart.p, nblk, norb, npr, norbs,
                                               sqrt((double)s0->electrons), (double *)dout.p);
    JCI_CUDA(cudaGetLastError());
    JCI_CUDA(cudaMemcpyAsync(dyorb, dout.p, sizeof(double) * (size_t)npr * norbs,
                             cudaMemcpyDeviceToHost, stm));
    JCI_CUDA(cudaStreamSynchronize(stm));
    return JCI_OK;
}
