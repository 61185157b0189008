// jci_io.cpp -- the reference's input/output formats, restated in C++.
//
//  * jayci.in namelists &general / &dalginfo (mpi_source/readnamelist.f90,
//    read through readgeninput / readdaiinput, ioutil.c:313,367) plus an
//    optional &gpuinfo block for this engine's own switches;
//  * SIFS integral files as readmoints.f90 consumes them (header 1 of
//    seven INTEGER*8, header 2, 1-e records decoded as colib sifd1 and
//    accumulated as sifr1n/sifrsh, 2-e records decoded as sifd2; 64-bit
//    dword with four 16-bit fields most-significant first (ulab16), 8-bit
//    orbital labels eight per word most-significant first (ulab8));
//  * unformatted vector files civec / ci.restart / hvvec (int32 dim, int32
//    len, dim*len float64; mpi_utilities.c:353-532);
//  * the Dyson-orbital program's dycicalc.in namelists &wavefcn0 /
//    &wavefcn1 / &dysonorbital (readnamelist.f90:110-180, ioutil.c:154-260)
//    and its dysonorb.dat output (run_pdycicalc.c:674-712).
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "jci_internal.h"

namespace {

std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

// Extract the body of namelist &name ... / (case-insensitive), comments
// (!) removed.  Returns false if the group is absent.
bool namelist_body(const std::string &text, const std::string &name, std::string &body) {
    std::string t;
    t.reserve(text.size());
    bool comment = false, quote = false;
    for (char c : text) {
        if (c == '\n') comment = false;
        if (c == '\'' || c == '"') quote = !quote;
        if (c == '!' && !quote) comment = true;
        if (!comment) t.push_back(c);
    }
    std::string lt = lower(t);
    std::string key = "&" + lower(name);
    size_t p = 0;
    while ((p = lt.find(key, p)) != std::string::npos) {
        size_t e = p + key.size();
        if (e < lt.size() && (std::isalnum((unsigned char)lt[e]) || lt[e] == '_')) {
            p = e;
            continue;
        }
        size_t end = lt.find('/', e);
        size_t end2 = lt.find("&end", e);
        if (end2 != std::string::npos && (end == std::string::npos || end2 < end)) end = end2;
        if (end == std::string::npos) return false;
        body = t.substr(e, end - e);
        return true;
    }
    return false;
}

bool parse_number(std::string v, double *out) {
    for (auto &c : v)
        if (c == 'd' || c == 'D') c = 'e';
    char *endp = nullptr;
    double x = strtod(v.c_str(), &endp);
    if (endp == v.c_str()) return false;
    while (*endp && std::isspace((unsigned char)*endp)) endp++;
    if (*endp) return false;
    *out = x;
    return true;
}

// key=value pairs separated by commas / whitespace.
bool parse_pairs(const std::string &body, std::vector<std::pair<std::string, std::string>> &kv) {
    size_t i = 0, n = body.size();
    while (i < n) {
        while (i < n && (std::isspace((unsigned char)body[i]) || body[i] == ',')) i++;
        if (i >= n) break;
        size_t k0 = i;
        while (i < n && body[i] != '=' && !std::isspace((unsigned char)body[i])) i++;
        std::string key = lower(body.substr(k0, i - k0));
        while (i < n && std::isspace((unsigned char)body[i])) i++;
        if (i >= n || body[i] != '=') return false;
        i++;
        while (i < n && std::isspace((unsigned char)body[i])) i++;
        size_t v0 = i;
        while (i < n && body[i] != ',' && !std::isspace((unsigned char)body[i])) i++;
        kv.emplace_back(key, body.substr(v0, i - v0));
    }
    return true;
}

// f10.5 output followed by %lf input, as the reference's restol takes
// (readnamelist.f90:105 "write(nmlstr(6),8) restol", 8 format(f10.5)).
double f10_5_roundtrip(double x) {
    char buf[64];
    snprintf(buf, sizeof(buf), "%10.5f", x);
    if (strlen(buf) > 10) return x;  // Fortran would print asterisks
    return atof(buf);
}

}  // namespace

extern "C" jci_status jci_read_namelists(const char *path, jci_general *g, jci_dalginfo *d,
                                         jci_gpuinfo *u) {
    if (!path) return JCI_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return JCI_ERR_IO;
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    fclose(f);
    std::string body;
    std::vector<std::pair<std::string, std::string>> kv;
    if (g) {
        // defaults of readnamelist.f90:69-76 (nactive has none: 0)
        *g = jci_general{0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (!namelist_body(text, "general", body) || !parse_pairs(body, kv)) return JCI_ERR_FORMAT;
        for (auto &p : kv) {
            double x;
            if (!parse_number(p.second, &x)) return JCI_ERR_FORMAT;
            int v = (int)x;
            if (p.first == "electrons") g->electrons = v;
            else if (p.first == "orbitals") g->orbitals = v;
            else if (p.first == "nfrozen") g->nfrozen = v;
            else if (p.first == "ndocc") g->ndocc = v;
            else if (p.first == "nactive") g->nactive = v;
            else if (p.first == "xlevel") g->xlevel = v;
            else if (p.first == "nfrzvirt") g->nfrzvirt = v;
            else if (p.first == "printlvl") g->printlvl = v;
            else if (p.first == "printwvf") g->printwvf = v;
            else return JCI_ERR_FORMAT;  // Fortran namelist read rejects unknown keys
        }
    }
    jci_gpuinfo gu{JCI_FP64, 1e-4, 0, 0};
    kv.clear();
    if (namelist_body(text, "gpuinfo", body)) {
        if (!parse_pairs(body, kv)) return JCI_ERR_FORMAT;
        for (auto &p : kv) {
            double x;
            if (!parse_number(p.second, &x)) return JCI_ERR_FORMAT;
            if (p.first == "precision") gu.precision = (int)x;
            else if (p.first == "switchtol") gu.switch_tol = x;
            else if (p.first == "block") gu.block = (int)x;
            else if (p.first == "exactrestol") gu.exact_restol = (int)x;
            else return JCI_ERR_FORMAT;
        }
    }
    if (u) *u = gu;
    if (d) {
        // defaults of readnamelist.f90:85-92
        *d = jci_dalginfo{20, 3, 8, 1, 1, 3, 1000, 1.0e-5};
        kv.clear();
        if (!namelist_body(text, "dalginfo", body) || !parse_pairs(body, kv))
            return JCI_ERR_FORMAT;
        for (auto &p : kv) {
            double x;
            if (!parse_number(p.second, &x)) return JCI_ERR_FORMAT;
            if (p.first == "maxiter") d->maxiter = (int)x;
            else if (p.first == "krymin") d->krymin = (int)x;
            else if (p.first == "krymax") d->krymax = (int)x;
            else if (p.first == "nroots") d->nroots = (int)x;
            else if (p.first == "prediagr") d->prediagr = (int)x;
            else if (p.first == "restol") d->restol = x;
            else if (p.first == "refdim") d->refdim = (int)x;
            else if (p.first == "buflen") d->buflen = (int)x;
            else return JCI_ERR_FORMAT;
        }
        if (!gu.exact_restol) d->restol = f10_5_roundtrip(d->restol);
    }
    return JCI_OK;
}

// ---- SIFS ----------------------------------------------------------------

namespace {

struct Reader {
    FILE *f;
    std::vector<unsigned char> rec;
    bool next() {
        int32_t a = 0, b = 0;
        if (fread(&a, 4, 1, f) != 1 || a < 0) return false;
        rec.resize((size_t)a);
        if (a && fread(rec.data(), 1, (size_t)a, f) != (size_t)a) return false;
        if (fread(&b, 4, 1, f) != 1 || b != a) return false;
        return true;
    }
    int64_t i64(size_t k) const {
        int64_t v;
        memcpy(&v, &rec[8 * k], 8);
        return v;
    }
    double f64(size_t k) const {
        double v;
        memcpy(&v, &rec[8 * k], 8);
        return v;
    }
    size_t words() const { return rec.size() / 8; }
};

struct Dword {
    int num, lab1, last, ifmt, itypea, itypeb, ibvtyp;
};

Dword unpack_dword(uint64_t w) {
    unsigned u1 = (unsigned)((w >> 48) & 0xffff), u2 = (unsigned)((w >> 32) & 0xffff);
    unsigned u3 = (unsigned)((w >> 16) & 0xffff), u4 = (unsigned)(w & 0xffff);
    Dword d;
    d.num = (int)u1;
    d.lab1 = (int)u2;
    d.last = (int)(u4 % 4);
    d.ifmt = (int)((u4 >> 2) % 8);
    d.itypeb = (int)(u3 % 1024);
    d.itypea = (int)((u3 >> 10) % 8);
    d.ibvtyp = (int)((u3 >> 13) % 8);
    return d;
}

uint64_t pack_dword(int num, int lab1, int itypea, int itypeb, int last, int ifmt) {
    uint64_t u1 = (uint64_t)num, u2 = (uint64_t)lab1;
    uint64_t u3 = (uint64_t)itypeb | ((uint64_t)itypea << 10);
    uint64_t u4 = (uint64_t)last | ((uint64_t)ifmt << 2);
    return (u1 << 48) | (u2 << 32) | (u3 << 16) | u4;
}

// 8-bit label k (0-based) of the packed label words starting at word w0
int label8(const Reader &r, size_t w0, long long k) {
    uint64_t w = (uint64_t)r.i64(w0 + k / 8);
    return (int)((w >> (56 - 8 * (k % 8))) & 0xff);
}

long long ix1(long long i, long long j) {
    return i > j ? (i - 1) * i / 2 + j : (j - 1) * j / 2 + i;
}

}  // namespace

// 2-e records (sifd2 with nipv = 4, colib8.f:447) from r into m2, until the
// record flagged last = 2.
static bool read_2e_records(Reader &r, long long l2rec, long long nbft, double *m2) {
    int last = 0;
    do {
        if (!r.next() || (long long)r.words() < l2rec) return false;
        Dword dw = unpack_dword((uint64_t)r.i64(0));
        last = dw.last;
        if (dw.ifmt != 0 || 1 + dw.num > (long long)r.words()) return false;
        for (int k = 0; k < dw.num; k++) {
            int l[4];
            for (int q = 0; q < 4; q++) l[q] = label8(r, dw.lab1 - 1, 4LL * k + q);
            for (int q = 0; q < 4; q++)
                if (l[q] < 1 || l[q] > nbft) return false;
            m2[ix1(ix1(l[0], l[1]), ix1(l[2], l[3])) - 1] += r.f64(1 + k);
        }
    } while (last != 2);
    return true;
}

static jci_status read_moints(const char *path, const char *path2, double *m1, long long m1cap,
                              double *m2, long long m2cap, int *nbft_out, double *nucrep,
                              double *frzcore) {
    if (!path || !m1 || !m2) return JCI_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return JCI_ERR_IO;
    Reader r{f, {}};
    jci_status st = JCI_ERR_FORMAT;
    do {
        // header 1 (readmoints.f90:101)
        if (!r.next() || r.words() < 7) break;
        long long ntitle = r.i64(1), nsym = r.i64(2), nbft = r.i64(3), ninfo = r.i64(4);
        long long nenrgy = r.i64(5), nmap = r.i64(6);
        if (nsym != 1 || nbft < 1 || nbft > 255 || ninfo < 6 || nenrgy < 1 || ntitle < 0 ||
            nmap < 0)
            break;  // symmetry-blocked files are not addressable by index1e
        long long n1 = ix1(nbft, nbft), n2 = ix1(n1, n1);
        if (n1 > m1cap || n2 > m2cap) {
            st = JCI_ERR_ARG;
            break;
        }
        // header 2 (readmoints.f90:299-332)
        if (!r.next()) break;
        size_t off = (size_t)ntitle * 80 + (size_t)nsym * 8 + (size_t)nsym * 4;
        if (r.rec.size() < off + (size_t)ninfo * 8 + nbft * 8 + nenrgy * 16) break;
        std::vector<int64_t> info(ninfo);
        memcpy(info.data(), &r.rec[off], ninfo * 8);
        off += (size_t)ninfo * 8 + (size_t)nbft * 8 + (size_t)nenrgy * 8;
        double e1;
        memcpy(&e1, &r.rec[off], 8);  // energy(1)
        long long l1rec = info[1], n1max = info[2], l2rec = info[3];
        // fsplit (info(1)): 1 = the 2-e records follow on this file; 2 = they
        // are on a second file (colib sifo2f, colib8.f:1720), which the
        // reference refuses (readmoints.f90:278-282) and this reader takes
        if (info[0] != 1 && info[0] != 2) break;
        if (info[5] != 0) break;  // only 8-bit label packing
        memset(m1, 0, sizeof(double) * m1cap);
        memset(m2, 0, sizeof(double) * m2cap);
        double hcore = 0.0;
        // 1-e records (sifr1n with btypes 0 -> S1, 1..6 -> H1)
        bool ok = true;
        int last = 0;
        do {
            if (!r.next() || (long long)r.words() < l1rec) {
                ok = false;
                break;
            }
            Dword dw = unpack_dword((uint64_t)r.i64(0));
            last = dw.last;
            if (dw.ifmt != 0 || dw.num > n1max || 2 + dw.num > (long long)r.words()) {
                ok = false;
                break;
            }
            bool h = dw.itypea == 0 && dw.itypeb >= 1 && dw.itypeb <= 6;
            if (h) {
                for (int k = 0; k < dw.num; k++) {
                    int a = label8(r, dw.lab1 - 1, 2LL * k), b = label8(r, dw.lab1 - 1, 2LL * k + 1);
                    if (a < 1 || b < 1 || a > nbft || b > nbft) {
                        ok = false;
                        break;
                    }
                    m1[ix1(a, b) - 1] += r.f64(1 + k);
                }
                if (dw.last != 0) hcore += r.f64(1 + dw.num);
            }
        } while (ok && last != 2);
        if (!ok) break;
        if (info[0] == 1) {
            if (!read_2e_records(r, l2rec, nbft, m2)) break;
        } else {
            // the second file holds only the 2-e records, one sequential
            // unformatted record of l2rec words each (colib aiopen/airead,
            // colib2.f:34,89)
            std::string p2 = path2 ? std::string(path2) : std::string(path) + "2";
            FILE *f2 = fopen(p2.c_str(), "rb");
            if (!f2) {
                st = JCI_ERR_IO;
                break;
            }
            Reader r2{f2, {}};
            ok = read_2e_records(r2, l2rec, nbft, m2);
            fclose(f2);
            if (!ok) break;
        }
        if (nbft_out) *nbft_out = (int)nbft;
        if (nucrep) *nucrep = e1;
        if (frzcore) *frzcore = hcore;
        st = JCI_OK;
    } while (0);
    fclose(f);
    return st;
}

extern "C" jci_status jci_read_moints(const char *path, double *m1, long long m1cap, double *m2,
                                      long long m2cap, int *nbft_out, double *nucrep,
                                      double *frzcore) {
    return read_moints(path, nullptr, m1, m1cap, m2, m2cap, nbft_out, nucrep, frzcore);
}

extern "C" jci_status jci_read_moints_split(const char *path, const char *path2, double *m1,
                                            long long m1cap, double *m2, long long m2cap,
                                            int *nbft_out, double *nucrep, double *frzcore) {
    if (!path2) return JCI_ERR_ARG;
    return read_moints(path, path2, m1, m1cap, m2, m2cap, nbft_out, nucrep, frzcore);
}

namespace {

struct Writer {
    FILE *f;
    bool rec(const void *p, size_t bytes) {
        int32_t n = (int32_t)bytes;
        return fwrite(&n, 4, 1, f) == 1 && (bytes == 0 || fwrite(p, 1, bytes, f) == bytes) &&
               fwrite(&n, 4, 1, f) == 1;
    }
};

void put_label8(std::vector<uint64_t> &buf, size_t w0, long long k, int v) {
    buf[w0 + k / 8] |= (uint64_t)(v & 0xff) << (56 - 8 * (k % 8));
}

}  // namespace

// fsplit 1 when path2 is null (every record on path), else 2 (the 2-e
// records on path2, as colib's sifew2 writes them through aiwrit).
static jci_status write_moints(const char *path, const char *path2, int nbft, const double *m1,
                               const double *m2, double nucrep, double frzcore) {
    if (!path || !m1 || !m2 || nbft < 1 || nbft > 255) return JCI_ERR_ARG;
    const long long l1rec = 4096, n1max = 3272, l2rec = 4096, n2max = 2730;
    FILE *f = fopen(path, "wb");
    if (!f) return JCI_ERR_IO;
    FILE *f2 = nullptr;
    if (path2 && !(f2 = fopen(path2, "wb"))) {
        fclose(f);
        return JCI_ERR_IO;
    }
    Writer w{f};
    bool ok = true;
    // header 1: version, ntitle, nsym, nbft, ninfo, nenrgy, nmap
    int64_t h1[7] = {2, 1, 1, nbft, 6, 1, 0};
    ok &= w.rec(h1, sizeof(h1));
    // header 2: title, nbpsy, slabel, info, bfnlab, ietype, energy
    std::vector<unsigned char> h2;
    auto put = [&](const void *p, size_t n) {
        const unsigned char *c = (const unsigned char *)p;
        h2.insert(h2.end(), c, c + n);
    };
    char title[81];
    snprintf(title, sizeof(title), "%-80s", "jci_b200 synthetic MO integrals");
    put(title, 80);
    int64_t nb = nbft;
    put(&nb, 8);
    put("a   ", 4);
    int64_t info[6] = {f2 ? 2 : 1, l1rec, n1max, l2rec, n2max, 0};
    put(info, sizeof(info));
    for (int i = 1; i <= nbft; i++) {
        char lab[9];
        snprintf(lab, sizeof(lab), "mo%-6d", i);
        put(lab, 8);
    }
    int64_t ietype = -1;  // nuclear repulsion
    put(&ietype, 8);
    put(&nucrep, 8);
    ok &= w.rec(h2.data(), h2.size());
    // 1-e arrays: S1 (identity, itypeb 0) then H1 (itypeb 6) with fcore
    long long n1 = ix1(nbft, nbft);
    for (int arr = 0; arr < 2 && ok; arr++) {
        std::vector<std::pair<long long, double>> vals;
        for (int i = 1; i <= nbft; i++)
            for (int j = 1; j <= i; j++) {
                double v = arr == 0 ? (i == j ? 1.0 : 0.0) : m1[ix1(i, j) - 1];
                if (v != 0.0) vals.push_back({(long long)i * 256 + j, v});
            }
        if (vals.empty()) vals.push_back({257, 0.0});
        size_t pos = 0;
        while (pos < vals.size()) {
            int num = (int)std::min<size_t>(n1max, vals.size() - pos);
            bool final_rec = pos + num == vals.size();
            int last = !final_rec ? 0 : (arr == 1 ? 2 : 1);
            std::vector<uint64_t> buf(l1rec, 0);
            int lab1 = num + 3;
            buf[0] = pack_dword(num, lab1, 0, arr == 0 ? 0 : 6, last, 0);
            for (int k = 0; k < num; k++) memcpy(&buf[1 + k], &vals[pos + k].second, 8);
            double fc = (arr == 1 && final_rec) ? frzcore : 0.0;
            memcpy(&buf[1 + num], &fc, 8);
            for (int k = 0; k < num; k++) {
                long long lab = vals[pos + k].first;
                put_label8(buf, lab1 - 1, 2LL * k, (int)(lab / 256));
                put_label8(buf, lab1 - 1, 2LL * k + 1, (int)(lab % 256));
            }
            ok &= w.rec(buf.data(), buf.size() * 8);
            pos += num;
        }
        (void)n1;
    }
    // 2-e records: each distinct (ij|kl), i>=j, k>=l, ij>=kl
    std::vector<std::pair<uint32_t, double>> v2;
    for (int i = 1; i <= nbft; i++)
        for (int j = 1; j <= i; j++)
            for (int k = 1; k <= i; k++)
                for (int l = 1; l <= k; l++) {
                    long long ij = ix1(i, j), kl = ix1(k, l);
                    if (kl > ij) continue;
                    double v = m2[ix1(ij, kl) - 1];
                    if (v == 0.0) continue;
                    v2.push_back({(uint32_t)(i << 24 | j << 16 | k << 8 | l), v});
                }
    if (v2.empty()) v2.push_back({(1u << 24) | (1u << 16) | (1u << 8) | 1u, 0.0});
    Writer w2{f2 ? f2 : f};
    size_t pos = 0;
    while (pos < v2.size() && ok) {
        int num = (int)std::min<size_t>(n2max, v2.size() - pos);
        int last = pos + num == v2.size() ? 2 : 0;
        std::vector<uint64_t> buf(l2rec, 0);
        int lab1 = num + 2;
        buf[0] = pack_dword(num, lab1, 3, 0, last, 0);
        for (int k = 0; k < num; k++) memcpy(&buf[1 + k], &v2[pos + k].second, 8);
        for (int k = 0; k < num; k++) {
            uint32_t lab = v2[pos + k].first;
            for (int q = 0; q < 4; q++)
                put_label8(buf, lab1 - 1, 4LL * k + q, (int)((lab >> (24 - 8 * q)) & 0xff));
        }
        ok &= w2.rec(buf.data(), buf.size() * 8);
        pos += num;
    }
    if (f2) ok &= fclose(f2) == 0;
    ok &= fclose(f) == 0;
    return ok ? JCI_OK : JCI_ERR_IO;
}

extern "C" jci_status jci_write_moints(const char *path, int nbft, const double *m1,
                                       const double *m2, double nucrep, double frzcore) {
    return write_moints(path, nullptr, nbft, m1, m2, nucrep, frzcore);
}

extern "C" jci_status jci_write_moints_split(const char *path, const char *path2, int nbft,
                                             const double *m1, const double *m2, double nucrep,
                                             double frzcore) {
    if (!path2) return JCI_ERR_ARG;
    return write_moints(path, path2, nbft, m1, m2, nucrep, frzcore);
}

// ---- vector files --------------------------------------------------------

extern "C" jci_status jci_write_vectors(const char *path, int dim, int len, const double *v) {
    if (!path || !v || dim < 0 || len < 0) return JCI_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return JCI_ERR_IO;
    bool ok = fwrite(&dim, sizeof(int), 1, f) == 1 && fwrite(&len, sizeof(int), 1, f) == 1 &&
              fwrite(v, sizeof(double), (size_t)dim * len, f) == (size_t)dim * len;
    ok &= fclose(f) == 0;
    return ok ? JCI_OK : JCI_ERR_IO;
}

extern "C" jci_status jci_read_vectors(const char *path, int dim, int len, double *v) {
    if (!path || !v || dim < 0 || len < 0) return JCI_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return JCI_ERR_IO;
    int fd = 0, fl = 0;
    jci_status st = JCI_OK;
    if (fread(&fd, sizeof(int), 1, f) != 1 || fread(&fl, sizeof(int), 1, f) != 1)
        st = JCI_ERR_FORMAT;
    else if (fd != dim || fl != len)  // read_gavectorsfile_dbl_ufmt error 5
        st = JCI_ERR_FORMAT;
    else if (fread(v, sizeof(double), (size_t)dim * len, f) != (size_t)dim * len)
        st = JCI_ERR_FORMAT;
    fclose(f);
    return st;
}

// ---- Dyson-orbital input and output -------------------------------------

namespace {

// key = value-list entries of a namelist body: "states0 = 1, 2" or
// "states0(2) = 3" (a 1-based element).  Values run up to the next key.
struct ListEntry {
    std::string key;
    int index;  // 0: whole array / scalar; else 1-based element
    std::vector<std::string> values;
};

bool parse_lists(const std::string &body, std::vector<ListEntry> &out) {
    std::vector<std::string> tok;
    std::string cur;
    for (char c : body) {
        if (std::isspace((unsigned char)c) || c == ',') {
            if (!cur.empty()) tok.push_back(cur);
            cur.clear();
        } else if (c == '=') {
            if (!cur.empty()) tok.push_back(cur);
            cur.clear();
            tok.push_back("=");
        } else {
            cur.push_back(c);
        }
    }
    if (!cur.empty()) tok.push_back(cur);
    for (size_t i = 0; i < tok.size();) {
        if (i + 1 >= tok.size() || tok[i + 1] != "=" || tok[i] == "=") return false;
        ListEntry e;
        std::string k = lower(tok[i]);
        e.index = 0;
        size_t lp = k.find('(');
        if (lp != std::string::npos) {
            size_t rp = k.find(')', lp);
            if (rp == std::string::npos) return false;
            e.index = atoi(k.substr(lp + 1, rp - lp - 1).c_str());
            if (e.index < 1) return false;
            k = k.substr(0, lp);
        }
        e.key = k;
        i += 2;
        while (i < tok.size() && tok[i] != "=" && !(i + 1 < tok.size() && tok[i + 1] == "="))
            e.values.push_back(tok[i++]);
        if (e.values.empty()) return false;
        out.push_back(e);
    }
    return true;
}

bool read_text(const char *path, std::string &text) {
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
    fclose(f);
    return true;
}

jci_status read_wavefcn(const std::string &text, const char *name, jci_wavefcn *w) {
    *w = jci_wavefcn{0, 0, 0, 0, 0, 0, 0, 0};
    std::string body;
    std::vector<ListEntry> kv;
    if (!namelist_body(text, name, body) || !parse_lists(body, kv)) return JCI_ERR_FORMAT;
    for (auto &e : kv) {
        double x;
        if (e.index || e.values.size() != 1 || !parse_number(e.values[0], &x))
            return JCI_ERR_FORMAT;
        int v = (int)x;
        if (e.key == "electrons") w->electrons = v;
        else if (e.key == "orbitals") w->orbitals = v;
        else if (e.key == "nfrozen") w->nfrozen = v;
        else if (e.key == "ndocc") w->ndocc = v;
        else if (e.key == "nactive") w->nactive = v;
        else if (e.key == "nfrzvirt") w->nfrzvirt = v;
        else if (e.key == "xlevel") w->xlevel = v;
        else if (e.key == "nstates") w->nstates = v;
        else return JCI_ERR_FORMAT;
    }
    return JCI_OK;
}

}  // namespace

extern "C" jci_status jci_read_dycicalc(const char *path, jci_wavefcn *wf0, jci_wavefcn *wf1,
                                        int *states0, int *nst0, int *states1, int *nst1) {
    if (!path || !wf0 || !wf1 || !states0 || !nst0 || !states1 || !nst1) return JCI_ERR_ARG;
    std::string text;
    if (!read_text(path, text)) return JCI_ERR_IO;
    jci_status r;
    if ((r = read_wavefcn(text, "wavefcn0", wf0))) return r;
    if ((r = read_wavefcn(text, "wavefcn1", wf1))) return r;
    // readnamelist.f90:164-165 defaults
    int s[2][5] = {{1, 0, 0, 0, 0}, {1, 0, 0, 0, 0}};
    std::string body;
    std::vector<ListEntry> kv;
    if (!namelist_body(text, "dysonorbital", body) || !parse_lists(body, kv))
        return JCI_ERR_FORMAT;
    for (auto &e : kv) {
        int w = e.key == "states0" ? 0 : e.key == "states1" ? 1 : -1;
        if (w < 0) return JCI_ERR_FORMAT;
        int first = e.index ? e.index - 1 : 0;
        if (first + (int)e.values.size() > 5) return JCI_ERR_FORMAT;
        for (size_t i = 0; i < e.values.size(); i++) {
            double x;
            if (!parse_number(e.values[i], &x)) return JCI_ERR_FORMAT;
            s[w][first + i] = (int)x;
        }
    }
    // ioutil.c:170-177: the count is the position of the last nonzero state
    *nst0 = *nst1 = 0;
    for (int i = 0; i < 5; i++) {
        states0[i] = s[0][i];
        states1[i] = s[1][i];
        if (s[0][i] != 0) *nst0 = i + 1;
        if (s[1][i] != 0) *nst1 = i + 1;
    }
    return JCI_OK;
}

extern "C" jci_status jci_write_dysonorb(const char *path, int ndyorbs, int orbs,
                                         const double *dyorb, const int *states0, int nst0,
                                         const int *states1, int nst1) {
    if (!path || !dyorb || !states0 || !states1 || ndyorbs < 0 || orbs < 0) return JCI_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return JCI_ERR_IO;
    fprintf(f, " %d %d %d\n", ndyorbs, nst0, nst1);
    fprintf(f, " %d\n", orbs);
    for (int i = 0; i < nst0; i++) fprintf(f, " %d", states0[i]);
    fprintf(f, "\n");
    for (int i = 0; i < nst1; i++) fprintf(f, " %d", states1[i]);
    fprintf(f, "\n");
    for (int i = 0; i < ndyorbs; i++) {
        for (int j = 0; j < orbs; j++) fprintf(f, "%15.8f\n", dyorb[(size_t)i * orbs + j]);
        fprintf(f, "\n");
    }
    return fclose(f) == 0 ? JCI_OK : JCI_ERR_IO;
}
