// jci_space.cpp -- truncated alpha/beta string space of the CI expansion.
//
// Builds, bit-exactly in the reference's order and addressing:
//   groups    allocate_eospace_array   (mpi_source/citruncate.c:121)
//   strings   generate_string_list     (citruncate.c:3971, :478 lexical
//             order DOCC-major, then ACTV, then VIRT sub-strings)
//   pairs     compute_detnum           (citruncate.c:414)
//   addresses occstr2address / str_adrfind (citruncate.c:4093,
//             straddress.c:48): lexical rank per sub-space, combined
//             DOCC-major and offset by the group start
//   phases    (-1)^(occupied orbitals strictly between io and fo)
//             (pindex_single_rep, action_util.c:1462); doubles multiply
//             the phase of io0->fo0 in the string by that of io1->fo1 in
//             the intermediate string (doublerep_cij_yij, citruncate.c:633)
// Every replacement whose result lies in the expansion is listed (the
// reference's generate_*x family, citruncate.c:755-3970, restricted per
// target group when queried).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "jci_internal.h"

namespace jci {

static long long g_binom[kMaxOrb + 2][kMaxElec + 2];
static std::once_flag g_binom_once;

static void init_binom() {
    std::call_once(g_binom_once, [] {
        for (int n = 0; n <= kMaxOrb + 1; n++)
            for (int k = 0; k <= kMaxElec + 1; k++) {
                if (k == 0) g_binom[n][k] = 1;
                else if (n == 0) g_binom[n][k] = 0;
                else g_binom[n][k] = g_binom[n - 1][k - 1] + g_binom[n - 1][k];
            }
    });
}

long long binom(int n, int k) {
    if (n < 0 || k < 0 || k > n) return 0;
    if (k > kMaxElec + 1 || n > kMaxOrb + 1) return 0;
    return g_binom[n][k];
}

// Groups in allocate_eospace_array order: DOCC electrons descending, ACTV
// electrons descending, VIRT electrons ascending.
static std::vector<Group> make_groups(int nelec, int norb, int ndocc,
                                      int nactv, int xlvl) {
    std::vector<Group> g;
    int vorbs = norb - ndocc - nactv;
    int mind = ndocc - std::min(ndocc, xlvl), maxd = ndocc;
    int mina = (nelec - ndocc) - std::min(nelec - ndocc, xlvl);
    int maxa = std::min(std::min(ndocc, xlvl) + (nelec - ndocc), nactv);
    for (int i = maxd; i >= mind; i--)
        for (int j = maxa; j >= mina; j--)
            for (int k = 0; k <= std::min(vorbs, xlvl); k++)
                if (i + j + k == nelec) g.push_back({i, j, k, 0, 0});
    return g;
}

// 0-based lexical rank of a sorted list r[0..e) of values in 1..m.
static long long lex_rank(const int *r, int e, int m) {
    long long a = 0;
    int prev = 0;
    for (int i = 1; i <= e; i++) {
        for (int j = prev + 1; j <= r[i - 1] - 1; j++) a += binom(m - j, e - i);
        prev = r[i - 1];
    }
    return a;
}

static bool lex_next(int *r, int e, int m) {
    for (int i = e - 1; i >= 0; i--)
        if (r[i] < m - (e - 1 - i)) {
            r[i]++;
            for (int j = i + 1; j < e; j++) r[j] = r[j - 1] + 1;
            return true;
        }
    return false;
}

static int find_group(const SpinSpace &sp, int d, int a, int v) {
    for (int g = 0; g < sp.ngrp; g++)
        if (sp.g[g].docc == d && sp.g[g].actv == a && sp.g[g].virt == v) return g;
    return -1;
}

int string_index(const jci_space *s, int spin, const int *o) {
    const SpinSpace &sp = s->sp[spin];
    int ne = sp.nelec, d = 0, a = 0, v = 0;
    for (int i = 0; i < ne; i++) {
        if (o[i] < 1 || o[i] > s->ci_orbs) return -1;
        if (i && o[i] <= o[i - 1]) return -1;
        if (o[i] <= s->ndocc) d++;
        else if (o[i] <= s->intorb) a++;
        else v++;
    }
    // check_istring (citruncate.c:225): enough DOCC, at most xlvl VIRT
    if (d < std::max(s->ndocc - s->xlvl, 0) || v > s->xlvl) return -1;
    int g = find_group(sp, d, a, v);
    if (g < 0) return -1;
    int vorb = s->ci_orbs - s->intorb;
    int rel[kMaxElec];
    for (int i = 0; i < d; i++) rel[i] = o[i];
    long long rd = lex_rank(rel, d, s->ndocc);
    for (int i = 0; i < a; i++) rel[i] = o[d + i] - s->ndocc;
    long long ra = lex_rank(rel, a, s->nactv);
    for (int i = 0; i < v; i++) rel[i] = o[d + a + i] - s->intorb;
    long long rv = lex_rank(rel, v, vorb);
    long long na = binom(s->nactv, a), nv = binom(vorb, v);
    return (int)(sp.g[g].start + (rd * na + ra) * nv + rv);
}

static void emit_group(const jci_space *s, SpinSpace &sp, const Group &g) {
    int ne = sp.nelec, vorb = s->ci_orbs - s->intorb;
    int dd[kMaxElec], aa[kMaxElec], vv[kMaxElec];
    for (int i = 0; i < g.docc; i++) dd[i] = i + 1;
    do {
        for (int i = 0; i < g.actv; i++) aa[i] = i + 1;
        do {
            for (int i = 0; i < g.virt; i++) vv[i] = i + 1;
            do {
                size_t base = sp.istr.size();
                sp.istr.resize(base + ne);
                int *o = &sp.istr[base];
                for (int i = 0; i < g.docc; i++) o[i] = dd[i];
                for (int i = 0; i < g.actv; i++) o[g.docc + i] = aa[i] + s->ndocc;
                for (int i = 0; i < g.virt; i++)
                    o[g.docc + g.actv + i] = vv[i] + s->intorb;
            } while (g.virt && lex_next(vv, g.virt, vorb));
        } while (g.actv && lex_next(aa, g.actv, s->nactv));
    } while (g.docc && lex_next(dd, g.docc, s->ndocc));
}

static inline int phase1(const int *o, int ne, int io, int fo) {
    int lo = std::min(io, fo), hi = std::max(io, fo), c = 0;
    for (int i = 0; i < ne; i++) c += (o[i] > lo && o[i] < hi);
    return (c & 1) ? -1 : 1;
}

static inline void replace_sorted(const int *o, int ne, int io, int fo, int *out) {
    int n = 0;
    for (int i = 0; i < ne; i++)
        if (o[i] != io) out[n++] = o[i];
    int k = n;
    while (k > 0 && out[k - 1] > fo) {
        out[k] = out[k - 1];
        k--;
    }
    out[k] = fo;
}

static void build_excitations(const jci_space *s, SpinSpace &sp, int spin) {
    int ne = sp.nelec, no = s->ci_orbs;
    sp.soff.assign(sp.nstr + 1, 0);
    sp.doff.assign(sp.nstr + 1, 0);
    sp.sing.clear();
    sp.doub.clear();
    sp.sing.reserve((size_t)sp.nstr * ne * (no - ne));
    std::vector<char> occ(no + 2);
    int t1[kMaxElec], t2[kMaxElec];
    for (int si = 0; si < sp.nstr; si++) {
        const int *o = &sp.istr[(size_t)si * ne];
        std::fill(occ.begin(), occ.end(), 0);
        for (int i = 0; i < ne; i++) occ[o[i]] = 1;
        sp.soff[si] = (long long)sp.sing.size();
        sp.doff[si] = (long long)sp.doub.size();
        // singles: electrons descending, targets ascending
        for (int e = ne - 1; e >= 0; e--)
            for (int f = 1; f <= no; f++) {
                if (occ[f]) continue;
                replace_sorted(o, ne, o[e], f, t1);
                int j = string_index(s, spin, t1);
                if (j < 0) continue;
                sp.sing.push_back({j, (int8_t)phase1(o, ne, o[e], f),
                                   (uint8_t)o[e], 0, (uint8_t)f, 0});
            }
        // doubles: electron pairs (e1 > e2) descending, target pairs ascending
        for (int e1 = ne - 1; e1 >= 1; e1--)
            for (int e2 = e1 - 1; e2 >= 0; e2--)
                for (int f1 = 1; f1 <= no; f1++) {
                    if (occ[f1]) continue;
                    replace_sorted(o, ne, o[e1], f1, t1);
                    int p1 = phase1(o, ne, o[e1], f1);
                    for (int f2 = f1 + 1; f2 <= no; f2++) {
                        if (occ[f2]) continue;
                        replace_sorted(t1, ne, o[e2], f2, t2);
                        int j = string_index(s, spin, t2);
                        if (j < 0) continue;
                        sp.doub.push_back({j, (int8_t)(p1 * phase1(t1, ne, o[e2], f2)),
                                           (uint8_t)o[e1], (uint8_t)o[e2],
                                           (uint8_t)f1, (uint8_t)f2});
                    }
                }
        sp.max_sing = std::max(sp.max_sing, (int)(sp.sing.size() - sp.soff[si]));
        sp.max_doub = std::max(sp.max_doub, (int)(sp.doub.size() - sp.doff[si]));
    }
    sp.soff[sp.nstr] = (long long)sp.sing.size();
    sp.doff[sp.nstr] = (long long)sp.doub.size();
}

jci_status finish_space(jci_space *s);

jci_status build_space(jci_space *s) {
    init_binom();
    // abecalc (abecalc.c:14): alpha gets the odd electron
    s->aelec = (s->electrons + 1) / 2;
    s->belec = s->electrons / 2;
    s->ci_aelec = s->aelec - s->nfrzc;
    s->ci_belec = s->belec - s->nfrzc;
    s->ci_orbs = s->orbitals - s->nfrzc - s->nfrzv;
    s->intorb = s->ndocc + s->nactv;
    if (s->electrons < 2 || s->ci_aelec < 1 || s->ci_belec < 1) return JCI_ERR_SPACE;
    if (s->ci_aelec > kMaxElec || s->ci_belec > kMaxElec) return JCI_ERR_SPACE;
    if (s->ci_orbs > kMaxOrb || s->intorb > kMaxInternal) return JCI_ERR_SPACE;
    if (s->ndocc < 0 || s->nactv < 1 || s->intorb > s->ci_orbs || s->xlvl < 0)
        return JCI_ERR_SPACE;
    int ne[2] = {s->ci_aelec, s->ci_belec};
    for (int spin = 0; spin < 2; spin++) {
        SpinSpace &sp = s->sp[spin];
        sp.nelec = ne[spin];
        sp.g = make_groups(ne[spin], s->ci_orbs, s->ndocc, s->nactv, s->xlvl);
        sp.ngrp = (int)sp.g.size();
        if (sp.ngrp == 0 || sp.ngrp > 20) return JCI_ERR_SPACE;
        int vorb = s->ci_orbs - s->intorb;
        long long tot = 0;
        for (auto &g : sp.g) {
            g.start = (int)tot;
            g.nstr = (int)(binom(s->ndocc, g.docc) * binom(s->nactv, g.actv) *
                           binom(vorb, g.virt));
            tot += g.nstr;
        }
        if (tot <= 0 || tot >= (1LL << 30)) return JCI_ERR_SPACE;
        sp.nstr = (int)tot;
        sp.istr.clear();
        sp.istr.reserve((size_t)tot * ne[spin]);
        sp.grp.assign(sp.nstr, 0);
        for (int gi = 0; gi < sp.ngrp; gi++) {
            emit_group(s, sp, sp.g[gi]);
            for (int i = 0; i < sp.g[gi].nstr; i++) sp.grp[sp.g[gi].start + i] = gi;
        }
    }
    // compute_detnum (citruncate.c:414-470)
    SpinSpace &P = s->sp[0], &Q = s->sp[1];
    int doccmin = std::max(2 * s->ndocc - s->xlvl, 0);
    int actvmin = std::max((s->ci_aelec - s->ndocc) + (s->ci_belec - s->ndocc) - s->xlvl, 0);
    s->pq.clear();
    s->pqoff.assign(1, 0);
    s->pairidx.assign((size_t)P.ngrp * Q.ngrp, -1);
    s->npq = 0;
    for (int i = 0; i < P.ngrp; i++)
        for (int j = 0; j < Q.ngrp; j++) {
            if (P.g[i].docc + Q.g[j].docc < doccmin) continue;
            if (P.g[i].actv + Q.g[j].actv < actvmin) continue;
            if (P.g[i].virt + Q.g[j].virt > s->xlvl) continue;
            s->pq.push_back(i);
            s->pq.push_back(j);
            s->pairidx[(size_t)i * Q.ngrp + j] = s->npq++;
            s->pqoff.push_back(s->pqoff.back() + (long long)P.g[i].nstr * Q.g[j].nstr);
        }
    s->ndets = s->pqoff.back();
    return finish_space(s);
}

// Excitation lists of both spins for a space whose strings, groups and
// pairs are set (shared by jci_space_create and the pdavidson drop-in).
jci_status finish_space(jci_space *s) {
    init_binom();
    if (s->ndets <= 0) return JCI_ERR_SPACE;
    try {
        for (int spin = 0; spin < 2; spin++) build_excitations(s, s->sp[spin], spin);
    } catch (const std::bad_alloc &) {
        return JCI_ERR_NOMEM;
    }
    return JCI_OK;
}

long long det_index(const jci_space *s, int p, int q) {
    int gp = s->sp[0].grp[p], gq = s->sp[1].grp[q];
    int k = s->pairidx[(size_t)gp * s->sp[1].ngrp + gq];
    if (k < 0) return -1;
    return s->pqoff[k] + (long long)(p - s->sp[0].g[gp].start) * s->sp[1].g[gq].nstr +
           (q - s->sp[1].g[gq].start);
}

void det_strings(const jci_space *s, long long d, int *pair, int *p, int *q) {
    int k = (int)(std::upper_bound(s->pqoff.begin(), s->pqoff.end(), d) - s->pqoff.begin()) - 1;
    const Group &gp = s->sp[0].g[s->pq[2 * k]];
    const Group &gq = s->sp[1].g[s->pq[2 * k + 1]];
    long long r = d - s->pqoff[k];
    *pair = k;
    *p = gp.start + (int)(r / gq.nstr);
    *q = gq.start + (int)(r % gq.nstr);
}

}  // namespace jci

using namespace jci;

extern "C" {

jci_status jci_space_create(int electrons, int orbitals, int nfrzc, int ndocc,
                            int nactv, int nfrzv, int xlvl, jci_space **out) {
    if (!out) return JCI_ERR_ARG;
    *out = nullptr;
    jci_space *s = new (std::nothrow) jci_space();
    if (!s) return JCI_ERR_NOMEM;
    s->electrons = electrons;
    s->orbitals = orbitals;
    s->nfrzc = nfrzc;
    s->ndocc = ndocc;
    s->nactv = nactv;
    s->nfrzv = nfrzv;
    s->xlvl = xlvl;
    jci_status st;
    try {
        st = build_space(s);
    } catch (const std::bad_alloc &) {
        st = JCI_ERR_NOMEM;
    }
    if (st != JCI_OK) {
        jci_space_destroy(s);
        return st;
    }
    *out = s;
    return JCI_OK;
}

void jci_space_destroy(jci_space *s) {
    if (!s) return;
    device_free(s);
    delete s;
}

jci_status jci_space_sizes(const jci_space *s, long long *out) {
    if (!s || !out) return JCI_ERR_ARG;
    out[0] = s->ci_aelec; out[1] = s->ci_belec; out[2] = s->ci_orbs;
    out[3] = s->sp[0].nstr; out[4] = s->sp[1].nstr;
    out[5] = s->sp[0].ngrp; out[6] = s->sp[1].ngrp;
    out[7] = s->npq; out[8] = s->ndets; out[9] = s->intorb;
    return JCI_OK;
}

jci_status jci_space_strings(const jci_space *s, int spin, int *istr) {
    if (!s || !istr || spin < 0 || spin > 1) return JCI_ERR_ARG;
    memcpy(istr, s->sp[spin].istr.data(), sizeof(int) * s->sp[spin].istr.size());
    return JCI_OK;
}

jci_status jci_space_eospaces(const jci_space *s, int spin, int *out) {
    if (!s || !out || spin < 0 || spin > 1) return JCI_ERR_ARG;
    const SpinSpace &sp = s->sp[spin];
    for (int g = 0; g < sp.ngrp; g++) {
        out[5 * g] = sp.g[g].docc;
        out[5 * g + 1] = sp.g[g].actv;
        out[5 * g + 2] = sp.g[g].virt;
        out[5 * g + 3] = sp.g[g].nstr;
        out[5 * g + 4] = sp.g[g].start;
    }
    return JCI_OK;
}

jci_status jci_space_pq(const jci_space *s, int *out) {
    if (!s || !out) return JCI_ERR_ARG;
    memcpy(out, s->pq.data(), sizeof(int) * s->pq.size());
    return JCI_OK;
}

jci_status jci_space_string_index(const jci_space *s, int spin, const int *orbs,
                                  int *index) {
    if (!s || !orbs || !index || spin < 0 || spin > 1) return JCI_ERR_ARG;
    *index = string_index(s, spin, orbs);
    return JCI_OK;
}

jci_status jci_space_excitations(const jci_space *s, int spin, int nrep, int istr,
                                 int teosp, int *out, int *count) {
    if (!s || !out || !count || spin < 0 || spin > 1 || (nrep != 1 && nrep != 2))
        return JCI_ERR_ARG;
    const SpinSpace &sp = s->sp[spin];
    if (istr < 0 || istr >= sp.nstr || teosp < 0 || teosp >= sp.ngrp) return JCI_ERR_ARG;
    const std::vector<long long> &off = nrep == 1 ? sp.soff : sp.doff;
    const std::vector<Exc> &lst = nrep == 1 ? sp.sing : sp.doub;
    int c = 0;
    for (long long k = off[istr]; k < off[istr + 1]; k++) {
        const Exc &e = lst[k];
        if (sp.grp[e.target] != teosp) continue;
        int *o = out + 6 * c++;
        o[0] = e.target; o[1] = e.io0; o[2] = e.io1;
        o[3] = e.fo0; o[4] = e.fo1; o[5] = e.sign;
    }
    *count = c;
    return JCI_OK;
}

}  // extern "C"
