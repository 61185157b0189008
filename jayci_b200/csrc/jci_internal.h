// jci_internal.h -- shared host-side types of libjci (not part of the ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "jci.h"

namespace jci {

constexpr int kMaxElec = 20;     // reference limit, execute_pjayci.c:145
constexpr int kMaxOrb = 200;     // reference limit, execute_pjayci.c:151
constexpr int kMaxInternal = 64; // ndocc + nactv, execute_pjayci.c:96

// One electron-occupation group of strings (struct eospace).
struct Group {
    int docc, actv, virt, nstr, start;
};

// A single or double replacement of a string.  Orbitals are 1-based.
struct Exc {
    int target;
    int8_t sign;
    uint8_t io0, io1, fo0, fo1;
};

struct SpinSpace {
    int nelec = 0, nstr = 0, ngrp = 0;
    std::vector<int> istr;  // nstr x nelec sorted 1-based orbital lists
    std::vector<int> grp;   // group of each string
    std::vector<Group> g;
    std::vector<long long> soff, doff;  // CSR offsets, nstr + 1
    std::vector<Exc> sing, doub;
    int max_sing = 0, max_doub = 0;
};

struct DeviceState;  // device tables and buffers (jci_device.cu)

}  // namespace jci

struct jci_space {
    int electrons = 0, orbitals = 0, nfrzc = 0, ndocc = 0, nactv = 0;
    int nfrzv = 0, xlvl = 0;
    int aelec = 0, belec = 0, ci_aelec = 0, ci_belec = 0, ci_orbs = 0;
    int intorb = 0;
    jci::SpinSpace sp[2];
    int npq = 0;
    std::vector<int> pq;          // npq x 2
    std::vector<int> pairidx;     // pegrps x qegrps -> pair or -1
    std::vector<long long> pqoff; // npq + 1
    long long ndets = 0;
    // integrals (host copies, packed as moindex.c)
    bool have_ints = false;
    std::vector<double> m1, m2;
    double nucrep = 0.0, frzcore = 0.0;
    jci::DeviceState *dev = nullptr;
};

namespace jci {

// Build strings / groups / pairs / excitation lists (jci_space.cpp).
jci_status build_space(jci_space *s);
long long binom(int n, int k);
int string_index(const jci_space *s, int spin, const int *orbs);
long long det_index(const jci_space *s, int p, int q);
void det_strings(const jci_space *s, long long d, int *pair, int *p, int *q);

// Device side (jci_device.cu).
jci_status device_init(jci_space *s);
jci_status device_set_integrals(jci_space *s);
void device_free(jci_space *s);
jci_status device_hdiag(jci_space *s, double *d_out);  // device pointer
jci_status device_sigma(jci_space *s, int nvec, const void *v, void *sig,
                        long long ld, int precision, void *stream);
float device_last_sigma_ms(jci_space *s);
jci_status davidson(jci_space *s, const jci_davidson_opts *o,
                    double *energies, double *civec, jci_davidson_stats *st);
jci_status davidson_vectors(jci_space *s, int k, double *out);

// I/O helpers (jci_io.cpp).
jci_status write_vectors(const char *path, int dim, int len, const double *v);

}  // namespace jci
