// jci_device.cu -- device tables, Hdiag and the generic sigma kernel.
//
// Matrix elements restate the reference's Slater rules
// (mpi_source/action_util.c):
//   hmatels_0x  :167  diagonal
//   hmatels_1x  :210  single, phase * [h(io,fo) + sum_{m in same, m != io}
//                     ((mm|io fo) - (m io|m fo)) + sum_{m in other} (mm|io fo)]
//   hmatels_2xaa:237  same-spin double, phase * [(i0 f0|i1 f1) - (i0 f1|i1 f0)]
//   hmatels_2xab:250  opposite-spin double, pa * pb * (ia fa|ib fb)
// The one-body part of every single (all but the opposite-spin sum) is
// tabulated once per integral set; the sigma kernels add the part that
// depends on the other string.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "jci_device.cuh"
#include "jci_kernels.cuh"

namespace jci {

jci_status cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    fprintf(stderr, "libjci: CUDA error %s (%s) at %s:%d: %s\n", cudaGetErrorName(e),
            cudaGetErrorString(e), file, line, what);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return JCI_ERR_NODEVICE;
    if (e == cudaErrorMemoryAllocation) return JCI_ERR_NOMEM;
    return JCI_ERR_CUDA;
}

template <typename T>
static jci_status upload(T **dst, const T *src, size_t n, cudaStream_t st) {
    if (n == 0) n = 1;
    JCI_CUDA(cudaMalloc((void **)dst, n * sizeof(T)));
    if (src) JCI_CUDA(cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return JCI_OK;
}

SpaceView make_view(const DeviceState *d) {
    SpaceView v;
    v.npq = d->npq;
    v.qegrps = d->t[1].ngrp;
    v.norb = d->norb;
    v.npair = d->npair;
    v.pqoff = d->pqoff;
    v.pairidx = d->pairidx;
    v.pqg = d->pqg;
    v.ndets = 0;
    v.skip = d->sigma_skip;
    const SpinTables *t[2] = {&d->t[0], &d->t[1]};
    SpaceView::Spin *o[2] = {&v.a, &v.b};
    for (int s = 0; s < 2; s++) {
        o[s]->nstr = t[s]->nstr;
        o[s]->nelec = t[s]->nelec;
        o[s]->istr = t[s]->istr;
        o[s]->grp = t[s]->grp;
        o[s]->gstart = t[s]->gstart;
        o[s]->gnstr = t[s]->gnstr;
        o[s]->soff = t[s]->soff;
        o[s]->doff = t[s]->doff;
        o[s]->sing = t[s]->sing;
        o[s]->doub = t[s]->doub;
    }
    return v;
}

jci_status device_init(jci_space *s) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return JCI_ERR_NODEVICE;
    }
    DeviceState *d = new (std::nothrow) DeviceState();
    if (!d) return JCI_ERR_NOMEM;
    s->dev = d;
    JCI_CUDA(cudaGetDevice(&d->device));
    JCI_CUDA(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
    JCI_CUDA(cudaEventCreate(&d->ev0));
    JCI_CUDA(cudaEventCreate(&d->ev1));
    JCI_CUDA(cudaEventCreateWithFlags(&d->evin, cudaEventDisableTiming));
    JCI_CUDA(cudaEventCreateWithFlags(&d->evout, cudaEventDisableTiming));
    d->norb = s->ci_orbs;
    d->npair = s->ci_orbs * (s->ci_orbs + 1) / 2;
    d->npq = s->npq;
    d->single_group = (s->sp[0].ngrp == 1 && s->sp[1].ngrp == 1);
    cudaStream_t st = d->stream;
    for (int spin = 0; spin < 2; spin++) {
        const SpinSpace &sp = s->sp[spin];
        SpinTables &t = d->t[spin];
        t.nstr = sp.nstr;
        t.nelec = sp.nelec;
        t.ngrp = sp.ngrp;
        t.max_sing = sp.max_sing;
        t.max_doub = sp.max_doub;
        t.nsing = (long long)sp.sing.size();
        t.ndoub = (long long)sp.doub.size();
        std::vector<int> gs(sp.ngrp), gn(sp.ngrp);
        for (int g = 0; g < sp.ngrp; g++) {
            gs[g] = sp.g[g].start;
            gn[g] = sp.g[g].nstr;
        }
        std::vector<uint2> sing(sp.sing.size()), doub(sp.doub.size());
        for (size_t k = 0; k < sp.sing.size(); k++) {
            const Exc &x = sp.sing[k];
            sing[k].x = (uint32_t)x.target | (x.sign < 0 ? 0x80000000u : 0u);
            sing[k].y = (uint32_t)x.io0 | ((uint32_t)x.fo0 << 8) |
                        ((uint32_t)pair_index(x.io0, x.fo0) << 16);
        }
        for (size_t k = 0; k < sp.doub.size(); k++) {
            const Exc &x = sp.doub[k];
            doub[k].x = (uint32_t)x.target | (x.sign < 0 ? 0x80000000u : 0u);
            doub[k].y = (uint32_t)x.io0 | ((uint32_t)x.fo0 << 8) |
                        ((uint32_t)x.io1 << 16) | ((uint32_t)x.fo1 << 24);
        }
        jci_status r;
        if ((r = upload(&t.istr, sp.istr.data(), sp.istr.size(), st))) return r;
        if ((r = upload(&t.grp, sp.grp.data(), sp.grp.size(), st))) return r;
        if ((r = upload(&t.gstart, gs.data(), gs.size(), st))) return r;
        if ((r = upload(&t.gnstr, gn.data(), gn.size(), st))) return r;
        if ((r = upload(&t.soff, sp.soff.data(), sp.soff.size(), st))) return r;
        if ((r = upload(&t.doff, sp.doff.data(), sp.doff.size(), st))) return r;
        if ((r = upload(&t.sing, sing.data(), sing.size(), st))) return r;
        if ((r = upload(&t.doub, doub.data(), doub.size(), st))) return r;
        if ((r = upload<double>(&t.a1, nullptr, sing.size(), st))) return r;
        if ((r = upload<float>(&t.a1f, nullptr, sing.size(), st))) return r;
        if ((r = upload<double>(&t.eself, nullptr, sp.nstr, st))) return r;
        // occupation masks (internal orbitals 1..64 -> bits 0..63)
        std::vector<uint64_t> occ(sp.nstr, 0);
        for (int i = 0; i < sp.nstr; i++)
            for (int e2 = 0; e2 < sp.nelec; e2++) {
                int o = sp.istr[(size_t)i * sp.nelec + e2];
                if (o <= 64) occ[i] |= 1ull << (o - 1);
            }
        if ((r = upload(&t.occ, occ.data(), occ.size(), st))) return r;
        if (d->single_group) {
            // dense [e][nstr] single tables: every string of a single group
            // has the same number of singles
            int ns = sp.max_sing;
            std::vector<uint32_t> fs((size_t)ns * sp.nstr);
            std::vector<uint16_t> fp((size_t)ns * sp.nstr);
            for (int i = 0; i < sp.nstr; i++)
                for (int k = 0; k < ns; k++) {
                    const uint2 &x = sing[sp.soff[i] + k];
                    fs[(size_t)k * sp.nstr + i] = x.x;
                    fp[(size_t)k * sp.nstr + i] = (uint16_t)(x.y >> 16);
                }
            if ((r = upload(&t.fsing, fs.data(), fs.size(), st))) return r;
            if ((r = upload(&t.fspair, fp.data(), fp.size(), st))) return r;
        }
    }
    jci_status r;
    if ((r = upload(&d->pairidx, s->pairidx.data(), s->pairidx.size(), st))) return r;
    if ((r = upload(&d->pqoff, s->pqoff.data(), s->pqoff.size(), st))) return r;
    if ((r = upload(&d->pqg, s->pq.data(), s->pq.size(), st))) return r;
    JCI_CUDA(cudaStreamSynchronize(st));
    return JCI_OK;
}

void device_free(jci_space *s) {
    DeviceState *d = s->dev;
    if (!d) return;
    cudaSetDevice(d->device);
    if (d->stream) cudaStreamSynchronize(d->stream);
    for (int spin = 0; spin < 2; spin++) {
        SpinTables &t = d->t[spin];
        void *p[] = {t.istr, t.grp, t.gstart, t.gnstr, t.soff, t.doff, t.sing, t.doub,
                     t.a1, t.a1f, t.eself, t.fsing, t.fspair, t.occ};
        for (void *q : p) cudaFree(q);
    }
    void *p[] = {d->pairidx, d->pqoff, d->pqg, d->m1, d->m2, d->m1f, d->m2f, d->hd,
                 d->hdf, d->io_v, d->io_s};
    for (void *q : p) cudaFree(q);
    fci_free(d);
    davidson_free(d);
    if (d->ev0) cudaEventDestroy(d->ev0);
    if (d->ev1) cudaEventDestroy(d->ev1);
    if (d->evin) cudaEventDestroy(d->evin);
    if (d->evout) cudaEventDestroy(d->evout);
    if (d->stream) cudaStreamDestroy(d->stream);
    delete d;
    s->dev = nullptr;
}

// ---- integral-dependent tables ------------------------------------------

// One-body part of every single replacement:
// h(io,fo) + sum_{m in string, m != io} ((mm|io fo) - (m io|m fo)).
__global__ void k_single_onebody(int nstr, int nelec, const int *__restrict__ istr,
                                 const long long *__restrict__ soff,
                                 const uint2 *__restrict__ sing,
                                 const double *__restrict__ m1,
                                 const double *__restrict__ m2, double *a1, float *a1f) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nstr) return;
    const int *o = istr + (long long)s * nelec;
    for (long long k = soff[s]; k < soff[s + 1]; k++) {
        uint2 x = sing[k];
        int io = x.y & 0xff, fo = (x.y >> 8) & 0xff, pr = x.y >> 16;
        double v = m1[pr];
        for (int e = 0; e < nelec; e++) {
            int m = o[e];
            if (m == io) continue;
            v += m2[eri_index(pair_index(m, m), pr)] -
                 m2[eri_index(pair_index(m, io), pair_index(m, fo))];
        }
        a1[k] = v;
        a1f[k] = (float)v;
    }
}

// Same-spin part of <i|H|i>: sum_a h_aa + sum_{a>b} ((aa|bb) - (ab|ab)).
__global__ void k_string_self(int nstr, int nelec, const int *__restrict__ istr,
                              const double *__restrict__ m1,
                              const double *__restrict__ m2, double *eself) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nstr) return;
    const int *o = istr + (long long)s * nelec;
    double v = 0.0;
    for (int i = 0; i < nelec; i++) {
        int a = o[i];
        v += m1[pair_index(a, a)];
        for (int j = 0; j < i; j++) {
            int b = o[j];
            v += m2[eri_index(pair_index(a, a), pair_index(b, b))] -
                 m2[eri_index(pair_index(a, b), pair_index(a, b))];
        }
    }
    eself[s] = v;
}

// <i|H|i> = self(alpha) + self(beta) + sum_{a in alpha, b in beta} (aa|bb)
// (hmatels_0x, action_util.c:167-201).
__global__ void k_hdiag(SpaceView v, const double *__restrict__ ea,
                        const double *__restrict__ eb, const double *__restrict__ m2,
                        double *hd, float *hdf) {
    long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= v.ndets) return;
    int k = 0;
    while (k + 1 < v.npq && v.pqoff[k + 1] <= d) k++;
    long long r = d - v.pqoff[k];
    int pg = v.pqg[2 * k], qg = v.pqg[2 * k + 1];
    int nq = v.b.gnstr[qg];
    int p = v.a.gstart[pg] + (int)(r / nq), q = v.b.gstart[qg] + (int)(r % nq);
    const int *oa = v.a.istr + (long long)p * v.a.nelec;
    const int *ob = v.b.istr + (long long)q * v.b.nelec;
    double x = ea[p] + eb[q];
    for (int i = 0; i < v.a.nelec; i++) {
        int pa = pair_index(oa[i], oa[i]);
        for (int j = 0; j < v.b.nelec; j++) x += m2[eri_index(pa, pair_index(ob[j], ob[j]))];
    }
    hd[d] = x;
    hdf[d] = (float)x;
}

template <typename T>
__global__ void k_convert(const double *__restrict__ in, T *out, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (T)in[i];
}

jci_status device_set_integrals(jci_space *s) {
    DeviceState *d = s->dev;
    JCI_CUDA(cudaSetDevice(d->device));
    cudaStream_t st = d->stream;
    long long m1len = (long long)d->npair, m2len = (long long)d->npair * (d->npair + 1) / 2;
    d->m2len = m2len;
    if (!d->m1) {
        JCI_CUDA(cudaMalloc(&d->m1, m1len * sizeof(double)));
        JCI_CUDA(cudaMalloc(&d->m2, m2len * sizeof(double)));
        JCI_CUDA(cudaMalloc(&d->m1f, m1len * sizeof(float)));
        JCI_CUDA(cudaMalloc(&d->m2f, m2len * sizeof(float)));
        JCI_CUDA(cudaMalloc(&d->hd, s->ndets * sizeof(double)));
        JCI_CUDA(cudaMalloc(&d->hdf, s->ndets * sizeof(float)));
    }
    JCI_CUDA(cudaMemcpyAsync(d->m1, s->m1.data(), m1len * sizeof(double),
                             cudaMemcpyHostToDevice, st));
    JCI_CUDA(cudaMemcpyAsync(d->m2, s->m2.data(), m2len * sizeof(double),
                             cudaMemcpyHostToDevice, st));
    k_convert<float><<<(unsigned)((m1len + 255) / 256), 256, 0, st>>>(d->m1, d->m1f, m1len);
    k_convert<float><<<(unsigned)((m2len + 255) / 256), 256, 0, st>>>(d->m2, d->m2f, m2len);
    for (int spin = 0; spin < 2; spin++) {
        SpinTables &t = d->t[spin];
        unsigned g = (unsigned)((t.nstr + 127) / 128);
        k_single_onebody<<<g, 128, 0, st>>>(t.nstr, t.nelec, t.istr, t.soff, t.sing, d->m1,
                                            d->m2, t.a1, t.a1f);
        k_string_self<<<g, 128, 0, st>>>(t.nstr, t.nelec, t.istr, d->m1, d->m2, t.eself);
    }
    SpaceView v = make_view(d);
    v.ndets = s->ndets;
    k_hdiag<<<(unsigned)((s->ndets + 255) / 256), 256, 0, st>>>(v, d->t[0].eself, d->t[1].eself,
                                                               d->m2, d->hd, d->hdf);
    JCI_CUDA(cudaGetLastError());
    jci_status r = fci_prepare(s);
    if (r != JCI_OK) return r;
    JCI_CUDA(cudaStreamSynchronize(st));
    return JCI_OK;
}

jci_status device_hdiag(jci_space *s, double *d_out) {
    DeviceState *d = s->dev;
    JCI_CUDA(cudaMemcpyAsync(d_out, d->hd, s->ndets * sizeof(double), cudaMemcpyDeviceToDevice,
                             d->stream));
    return JCI_OK;
}

// ---- generic sigma ------------------------------------------------------
//
// One thread per determinant i = (pair, p, q); a full-row gather over every
// determinant j connected to i by the Slater rules (both triangles), so each
// sigma element is written exactly once and no atomics are needed.

__device__ __forceinline__ long long view_det(const SpaceView &v, int p, int q) {
    int gp = v.a.grp[p], gq = v.b.grp[q];
    int k = v.pairidx[gp * v.qegrps + gq];
    if (k < 0) return -1;
    return v.pqoff[k] + (long long)(p - v.a.gstart[gp]) * v.b.gnstr[gq] + (q - v.b.gstart[gq]);
}

template <typename T>
__device__ __forceinline__ T coul_other(const int *o, int ne, int pr, const T *m2) {
    T s = 0;
    for (int e = 0; e < ne; e++) s += m2[eri_index(pair_index(o[e], o[e]), pr)];
    return s;
}

template <typename T, int NV>
__global__ void __launch_bounds__(128) k_sigma_generic(SpaceView v, const T *__restrict__ hd,
                                                       const T *__restrict__ m2,
                                                       const T *__restrict__ a1a,
                                                       const T *__restrict__ a1b,
                                                       const T *__restrict__ V, T *__restrict__ S,
                                                       long long ld, int nvec) {
    long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= v.ndets || (v.skip && *v.skip)) return;
    int k = 0;
    while (k + 1 < v.npq && v.pqoff[k + 1] <= d) k++;
    int pg = v.pqg[2 * k], qg = v.pqg[2 * k + 1];
    long long r = d - v.pqoff[k];
    int nq = v.b.gnstr[qg];
    int p = v.a.gstart[pg] + (int)(r / nq), q = v.b.gstart[qg] + (int)(r % nq);
    const int *oa = v.a.istr + (long long)p * v.a.nelec;
    const int *ob = v.b.istr + (long long)q * v.b.nelec;
    T acc[NV];
    T hdd = hd[d];
#pragma unroll
    for (int c = 0; c < NV; c++) acc[c] = c < nvec ? hdd * V[c * ld + d] : T(0);
    // alpha singles (same beta) and alpha x beta singles
    for (long long e = v.a.soff[p]; e < v.a.soff[p + 1]; e++) {
        uint2 x = v.a.sing[e];
        int tgt = x.x & 0x3fffffff;
        T sa = (x.x >> 31) ? T(-1) : T(1);
        int pra = x.y >> 16;
        long long j = view_det(v, tgt, q);
        if (j >= 0) {
            T h = sa * (a1a[e] + coul_other(ob, v.b.nelec, pra, m2));
#pragma unroll
            for (int c = 0; c < NV; c++)
                if (c < nvec) acc[c] += h * V[c * ld + j];
        }
        for (long long f = v.b.soff[q]; f < v.b.soff[q + 1]; f++) {
            uint2 y = v.b.sing[f];
            long long jj = view_det(v, tgt, y.x & 0x3fffffff);
            if (jj < 0) continue;
            T h = ((y.x >> 31) ? -sa : sa) * m2[eri_index(pra, y.y >> 16)];
#pragma unroll
            for (int c = 0; c < NV; c++)
                if (c < nvec) acc[c] += h * V[c * ld + jj];
        }
    }
    // alpha doubles
    for (long long e = v.a.doff[p]; e < v.a.doff[p + 1]; e++) {
        uint2 x = v.a.doub[e];
        long long j = view_det(v, x.x & 0x3fffffff, q);
        if (j < 0) continue;
        int i0 = x.y & 0xff, f0 = (x.y >> 8) & 0xff, i1 = (x.y >> 16) & 0xff, f1 = x.y >> 24;
        T h = m2[eri_index(pair_index(i0, f0), pair_index(i1, f1))] -
              m2[eri_index(pair_index(i0, f1), pair_index(i1, f0))];
        if (x.x >> 31) h = -h;
#pragma unroll
        for (int c = 0; c < NV; c++)
            if (c < nvec) acc[c] += h * V[c * ld + j];
    }
    // beta singles (same alpha)
    for (long long f = v.b.soff[q]; f < v.b.soff[q + 1]; f++) {
        uint2 y = v.b.sing[f];
        long long j = view_det(v, p, y.x & 0x3fffffff);
        if (j < 0) continue;
        T h = a1b[f] + coul_other(oa, v.a.nelec, y.y >> 16, m2);
        if (y.x >> 31) h = -h;
#pragma unroll
        for (int c = 0; c < NV; c++)
            if (c < nvec) acc[c] += h * V[c * ld + j];
    }
    // beta doubles
    for (long long f = v.b.doff[q]; f < v.b.doff[q + 1]; f++) {
        uint2 y = v.b.doub[f];
        long long j = view_det(v, p, y.x & 0x3fffffff);
        if (j < 0) continue;
        int i0 = y.y & 0xff, f0 = (y.y >> 8) & 0xff, i1 = (y.y >> 16) & 0xff, f1 = y.y >> 24;
        T h = m2[eri_index(pair_index(i0, f0), pair_index(i1, f1))] -
              m2[eri_index(pair_index(i0, f1), pair_index(i1, f0))];
        if (y.x >> 31) h = -h;
#pragma unroll
        for (int c = 0; c < NV; c++)
            if (c < nvec) acc[c] += h * V[c * ld + j];
    }
#pragma unroll
    for (int c = 0; c < NV; c++)
        if (c < nvec) S[c * ld + d] = acc[c];
}

template <typename T>
static void launch_generic(const DeviceState *dv, long long ndets, const T *hd, const T *m2,
                           const T *a1a, const T *a1b, const T *V, T *S, long long ld,
                           int nvec, cudaStream_t st) {
    SpaceView v = make_view(dv);
    v.ndets = ndets;
    unsigned grid = (unsigned)((ndets + 127) / 128);
    for (int c0 = 0; c0 < nvec; c0 += 4) {
        int nv = std::min(4, nvec - c0);
        k_sigma_generic<T, 4><<<grid, 128, 0, st>>>(v, hd, m2, a1a, a1b, V + c0 * ld,
                                                   S + c0 * ld, ld, nv);
    }
}

jci_status device_sigma(jci_space *s, int nvec, const void *vin, void *sout, long long ld,
                        int precision, void *stream) {
    DeviceState *d = s->dev;
    if (!s->have_ints) return JCI_ERR_STATE;
    if (nvec < 1 || ld < s->ndets || !vin || !sout) return JCI_ERR_ARG;
    cudaStream_t st = stream ? (cudaStream_t)stream : d->stream;
    // no timing events while the stream is being captured into a graph
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    JCI_CUDA(cudaStreamIsCapturing(st, &cap));
    const bool timed = cap == cudaStreamCaptureStatusNone;
    if (timed) JCI_CUDA(cudaEventRecord(d->ev0, st));
    jci_status r = JCI_OK;
    if (d->single_group && fci_supported(s)) {
        r = fci_sigma(s, nvec, vin, sout, ld, precision, st);
    } else if (precision == JCI_FP32) {
        launch_generic<float>(d, s->ndets, d->hdf, d->m2f, d->t[0].a1f, d->t[1].a1f,
                              (const float *)vin, (float *)sout, ld, nvec, st);
    } else {
        launch_generic<double>(d, s->ndets, d->hd, d->m2, d->t[0].a1, d->t[1].a1,
                               (const double *)vin, (double *)sout, ld, nvec, st);
    }
    if (r != JCI_OK) return r;
    JCI_CUDA(cudaGetLastError());
    if (timed) JCI_CUDA(cudaEventRecord(d->ev1, st));
    return JCI_OK;
}

// Generic path only (used by tests to cross-check the FCI kernels).
jci_status device_sigma_generic(jci_space *s, int nvec, const void *vin, void *sout,
                                long long ld, int precision, cudaStream_t st) {
    DeviceState *d = s->dev;
    if (precision == JCI_FP32)
        launch_generic<float>(d, s->ndets, d->hdf, d->m2f, d->t[0].a1f, d->t[1].a1f,
                              (const float *)vin, (float *)sout, ld, nvec, st);
    else
        launch_generic<double>(d, s->ndets, d->hd, d->m2, d->t[0].a1, d->t[1].a1,
                               (const double *)vin, (double *)sout, ld, nvec, st);
    JCI_CUDA(cudaGetLastError());
    return JCI_OK;
}

float device_last_sigma_ms(jci_space *s) {
    DeviceState *d = s->dev;
    float ms = 0.f;
    cudaEventSynchronize(d->ev1);
    cudaEventElapsedTime(&ms, d->ev0, d->ev1);
    return ms;
}

}  // namespace jci
