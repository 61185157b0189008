// jci_api.cpp -- C ABI entry points of libjci (declared in include/jci.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "jci_internal.h"
#include "jci_kernels.cuh"

namespace jci {
jci_status finish_space(jci_space *s);
}

using namespace jci;

extern "C" {

const char *jci_status_string(int st) {
    switch (st) {
        case JCI_OK: return "ok";
        case JCI_ERR_ARG: return "invalid argument";
        case JCI_ERR_SPACE: return "CI space outside the supported limits";
        case JCI_ERR_NOMEM: return "out of memory";
        case JCI_ERR_CUDA: return "CUDA runtime error";
        case JCI_ERR_NODEVICE: return "no CUDA device (libjci has no CPU fallback)";
        case JCI_ERR_IO: return "file I/O error";
        case JCI_ERR_FORMAT: return "malformed input file";
        case JCI_ERR_NOCONV: return "Davidson did not converge within maxiter";
        case JCI_ERR_LINALG: return "subspace eigensolve failed";
        case JCI_ERR_TIMEOUT: return "bounded device wait expired";
        case JCI_ERR_BUSY: return "server admission refused";
        case JCI_ERR_STATE: return "call out of order";
        default: return "unknown status";
    }
}

int jci_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

jci_status jci_set_integrals(jci_space *s, const double *m1, const double *m2, int norb,
                             double nucrep, double frzcore) {
    if (!s || !m1 || !m2) return JCI_ERR_ARG;
    if (norb != s->ci_orbs) return JCI_ERR_ARG;
    long long n1 = (long long)norb * (norb + 1) / 2, n2 = n1 * (n1 + 1) / 2;
    try {
        s->m1.assign(m1, m1 + n1);
        s->m2.assign(m2, m2 + n2);
    } catch (const std::bad_alloc &) {
        return JCI_ERR_NOMEM;
    }
    s->nucrep = nucrep;
    s->frzcore = frzcore;
    jci_status r = JCI_OK;
    if (!s->dev) r = device_init(s);  // device tables are built on first use
    if (r) return r;
    r = device_set_integrals(s);
    if (r) return r;
    s->have_ints = true;
    return JCI_OK;
}

jci_status jci_hdiag(jci_space *s, double *out) {
    if (!s || !out) return JCI_ERR_ARG;
    if (!s->have_ints) return JCI_ERR_STATE;
    double *d = nullptr;
    if (cudaMalloc(&d, s->ndets * sizeof(double)) != cudaSuccess) return JCI_ERR_NOMEM;
    jci_status r = device_hdiag(s, d);
    if (!r && cudaMemcpy(out, d, s->ndets * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        r = JCI_ERR_CUDA;
    cudaFree(d);
    return r;
}

jci_status jci_sigma_device(jci_space *s, int nvec, const void *v, void *sig, long long ld,
                            int precision, void *stream) {
    if (!s) return JCI_ERR_ARG;
    if (precision != JCI_FP64 && precision != JCI_FP32) return JCI_ERR_ARG;
    if (stream || !s->dev) return device_sigma(s, nvec, v, sig, ld, precision, stream);
    // NULL stream: the handle's stream, after the work the caller queued on
    // the legacy default stream (its inputs and outputs are often written
    // there), and that stream waits for the sigma
    DeviceState *d = s->dev;
    JCI_CUDA(cudaEventRecord(d->evin, cudaStreamLegacy));
    JCI_CUDA(cudaStreamWaitEvent(d->stream, d->evin, 0));
    jci_status r = device_sigma(s, nvec, v, sig, ld, precision, nullptr);
    if (r) return r;
    JCI_CUDA(cudaEventRecord(d->evout, d->stream));
    JCI_CUDA(cudaStreamWaitEvent(cudaStreamLegacy, d->evout, 0));
    return JCI_OK;
}

jci_status jci_sigma(jci_space *s, int nvec, const double *v, double *sig, int precision) {
    if (!s || !v || !sig || nvec < 1) return JCI_ERR_ARG;
    if (precision != JCI_FP64 && precision != JCI_FP32) return JCI_ERR_ARG;
    if (!s->have_ints) return JCI_ERR_STATE;
    long long n = s->ndets;
    size_t w = precision == JCI_FP32 ? sizeof(float) : sizeof(double);
    size_t bytes = (size_t)nvec * n * w;
    DeviceState *d = s->dev;
    cudaStream_t st = d->stream;
    // staging buffers stay with the handle (grown on demand)
    if (d->io_bytes < bytes) {
        cudaFree(d->io_v);
        cudaFree(d->io_s);
        d->io_v = d->io_s = nullptr;
        d->io_bytes = 0;
        if (cudaMalloc(&d->io_v, bytes) != cudaSuccess) return JCI_ERR_NOMEM;
        if (cudaMalloc(&d->io_s, bytes) != cudaSuccess) return JCI_ERR_NOMEM;
        d->io_bytes = bytes;
    }
    jci_status r = JCI_OK;
    std::vector<float> tmp;
    if (precision == JCI_FP32) {
        tmp.resize((size_t)nvec * n);
        for (size_t i = 0; i < tmp.size(); i++) tmp[i] = (float)v[i];
        if (cudaMemcpyAsync(d->io_v, tmp.data(), bytes, cudaMemcpyHostToDevice, st))
            r = JCI_ERR_CUDA;
    } else if (cudaMemcpyAsync(d->io_v, v, bytes, cudaMemcpyHostToDevice, st)) {
        r = JCI_ERR_CUDA;
    }
    if (!r) r = device_sigma(s, nvec, d->io_v, d->io_s, n, precision, nullptr);
    if (!r) {
        void *dst = precision == JCI_FP32 ? (void *)tmp.data() : (void *)sig;
        if (cudaMemcpyAsync(dst, d->io_s, bytes, cudaMemcpyDeviceToHost, st)) r = JCI_ERR_CUDA;
    }
    if (!r && cudaStreamSynchronize(st) != cudaSuccess) r = JCI_ERR_CUDA;
    if (!r) r = fci_wait_status(s);
    if (!r && precision == JCI_FP32)
        for (size_t i = 0; i < tmp.size(); i++) sig[i] = tmp[i];
    return r;
}

jci_status jci_sigma_tuning(const jci_space *s, int precision, int *mode, int *threads,
                            int *rows, int *batch, float *ms) {
    if (!s || !mode || !threads || !rows || !batch || !ms) return JCI_ERR_ARG;
    fci_tuning(s, precision, mode, threads, rows, batch, ms);
    return JCI_OK;
}

jci_status jci_sigma_device_noalloc(jci_space *s, const void *v, void *sig, int precision,
                                    void *stream) {
    if (!s || !v || !sig) return JCI_ERR_ARG;
    if (precision != JCI_FP64 && precision != JCI_FP32) return JCI_ERR_ARG;
    if (!s->have_ints || !s->dev) return JCI_ERR_STATE;
    if (cudaSetDevice(s->dev->device) != cudaSuccess) return JCI_ERR_CUDA;
    cudaStream_t st = stream ? (cudaStream_t)stream : s->dev->stream;
    return fci_sigma_noalloc(s, v, sig, precision, st);
}

jci_status jci_sigma_set_plan(jci_space *s, int precision, int mode, int threads, int rows,
                              int batch) {
    if (!s || (precision != JCI_FP64 && precision != JCI_FP32) || mode < 0 || mode > 7)
        return JCI_ERR_ARG;
    if (!s->have_ints) return JCI_ERR_STATE;
    return fci_force_plan(s, precision, mode, threads, rows, batch);
}

jci_status jci_test_expire_next_wait(jci_space *s) {
    if (!s) return JCI_ERR_ARG;
    if (!s->have_ints || !fci_supported(s)) return JCI_ERR_STATE;
    return fci_arm_wait_expiry(s);
}

void jci_davidson_defaults(jci_davidson_opts *o) {
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->maxiter = 20;
    o->krymin = 3;
    o->krymax = 8;
    o->nroots = 1;
    o->prediagr = 1;
    o->refdim = 3;
    o->restol = 1e-5;
    o->precision = JCI_FP64;
    o->switch_tol = 1e-4;
}

jci_status jci_davidson(jci_space *s, const jci_davidson_opts *o, double *energies,
                        double *civec, jci_davidson_stats *st) {
    if (!s || !o || !energies) return JCI_ERR_ARG;
    if (o->precision != JCI_FP64 && o->precision != JCI_MIXED) return JCI_ERR_ARG;
    if (o->prediagr < 1 || o->prediagr > 3) return JCI_ERR_ARG;
    return davidson(s, o, energies, civec, st);
}

// Drop-in replacement of the reference's pdavidson (pdavidson.h:9).  The
// space is rebuilt from the caller's citrunc output: string orbital lists,
// groups and (p,q) pairs are taken as given, the excitation lists are
// regenerated.
int jci_pdavidson(struct jci_occstr *pstrings, struct jci_eospace *peospace, int pegrps,
                  struct jci_occstr *qstrings, struct jci_eospace *qeospace, int qegrps,
                  int **pq_space_pairs, int num_pq, double *moints1, double *moints2,
                  int aelec, int belec, int intorb, int ndets, double nucrep_e,
                  double frzcore_e, int printlvl, int maxiter, int krymin, int krymax,
                  int nroots, int prediagr, int refdim, double restol, int ga_buffer_len,
                  int nmos, int ndocc, int nactv) {
    (void)ga_buffer_len;
    if (!pstrings || !peospace || !qstrings || !qeospace || !pq_space_pairs || !moints1 ||
        !moints2)
        return JCI_ERR_ARG;
    if (aelec < 1 || belec < 1 || aelec > kMaxElec || belec > kMaxElec || nmos > kMaxOrb ||
        intorb != ndocc + nactv || pegrps < 1 || qegrps < 1 || pegrps > 20 || qegrps > 20)
        return JCI_ERR_SPACE;
    jci_space *s = new (std::nothrow) jci_space();
    if (!s) return JCI_ERR_NOMEM;
    s->ci_aelec = aelec;
    s->ci_belec = belec;
    s->ci_orbs = nmos;
    s->ndocc = ndocc;
    s->nactv = nactv;
    s->intorb = intorb;
    s->xlvl = kMaxElec;  // groups and pairs are given; membership decides
    s->electrons = aelec + belec;
    s->orbitals = nmos;
    struct jci_occstr *str[2] = {pstrings, qstrings};
    struct jci_eospace *eo[2] = {peospace, qeospace};
    int ng[2] = {pegrps, qegrps}, ne[2] = {aelec, belec};
    jci_status r = JCI_OK;
    for (int spin = 0; spin < 2 && !r; spin++) {
        SpinSpace &sp = s->sp[spin];
        sp.nelec = ne[spin];
        sp.ngrp = ng[spin];
        long long tot = 0;
        for (int g = 0; g < ng[spin]; g++) {
            const jci_eospace &e = eo[spin][g];
            if (e.start != tot || e.nstr < 0) r = JCI_ERR_ARG;
            sp.g.push_back({e.docc, e.actv, e.virt, e.nstr, e.start});
            tot += e.nstr;
        }
        sp.nstr = (int)tot;
        sp.istr.resize((size_t)tot * ne[spin]);
        sp.grp.assign((size_t)tot, 0);
        for (int g = 0; g < ng[spin]; g++)
            for (int i = 0; i < eo[spin][g].nstr; i++) sp.grp[eo[spin][g].start + i] = g;
        for (long long i = 0; i < tot; i++)
            for (int k = 0; k < ne[spin]; k++)
                sp.istr[(size_t)i * ne[spin] + k] = str[spin][i].istr[k];
    }
    if (!r) {
        s->npq = num_pq;
        s->pqoff.assign(1, 0);
        s->pairidx.assign((size_t)pegrps * qegrps, -1);
        for (int k = 0; k < num_pq; k++) {
            int p = pq_space_pairs[k][0], q = pq_space_pairs[k][1];
            if (p < 0 || p >= pegrps || q < 0 || q >= qegrps) {
                r = JCI_ERR_ARG;
                break;
            }
            s->pq.push_back(p);
            s->pq.push_back(q);
            s->pairidx[(size_t)p * qegrps + q] = k;
            s->pqoff.push_back(s->pqoff.back() +
                               (long long)peospace[p].nstr * qeospace[q].nstr);
        }
        s->ndets = s->pqoff.back();
        if (s->ndets != ndets) r = JCI_ERR_ARG;
    }
    if (!r) r = finish_space(s);
    if (!r) r = jci_set_integrals(s, moints1, moints2, nmos, nucrep_e, frzcore_e);
    std::vector<double> e(std::max(nroots, 1));
    if (!r) {
        jci_davidson_opts o;
        jci_davidson_defaults(&o);
        o.maxiter = maxiter;
        o.krymin = krymin;
        o.krymax = krymax;
        o.nroots = nroots;
        o.prediagr = prediagr;
        o.refdim = refdim;
        o.restol = restol;
        o.printlvl = printlvl;
        o.write_files = 1;
        jci_davidson_stats st;
        r = davidson(s, &o, e.data(), nullptr, &st);
        if (printlvl >= 0 && (r == JCI_OK || r == JCI_ERR_NOCONV)) {
            for (int k = 0; k < nroots; k++) printf("   Root #%2d  %18.10lf\n", k + 1, e[k]);
            printf(" Davidson algorithm finished (%s). \n",
                   r == JCI_OK ? "converged" : "not converged");
            fflush(stdout);
        }
        if (r == JCI_ERR_NOCONV) r = JCI_OK;  // the reference returns 0 here too
    }
    jci_space_destroy(s);
    return (int)r;
}

}  // extern "C"
