/*
 * jci.h -- C ABI of libjci, the B200-native determinant-CI engine.
 *
 * Drop-in boundary for the JayCI hot path: the truncated alpha/beta string
 * space, the direct Slater-rule sigma = H c build and the Davidson
 * eigensolver around it.  All compute runs on the current CUDA device;
 * there is no CPU fallback (calls fail with JCI_ERR_NODEVICE / JCI_ERR_CUDA).
 *
 * Signatures use plain C types only.  Citations name the reference
 * interface each entry point replaces (paths within the JayCI project).
 *
 * Conventions shared with the reference:
 *  - orbitals are 1-based; strings are sorted orbital lists;
 *  - determinants are ordered by (p,q)-group pair, then alpha string, then
 *    beta string (pdavidson.c:4757 string_info_to_determinant_fast);
 *  - integrals are packed as in moindex.c: moints1[index1e(i,j)-1],
 *    moints2[index2e(i,j,k,l)-1] with index1e(i,j) = max(i,j)(max-1)/2+min;
 *  - vectors are stored vector-major: v[k*ndets + i].
 *
 * Thread safety: distinct handles may be used from distinct host threads;
 * one handle must not be used concurrently.  Every call returns a status;
 * the library never exits the process.
 */
#ifndef JCI_H
#define JCI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
        JCI_OK = 0,
        JCI_ERR_ARG = 1,       /* invalid argument */
        JCI_ERR_SPACE = 2,     /* CI space outside the supported limits */
        JCI_ERR_NOMEM = 3,     /* host or device allocation failed */
        JCI_ERR_CUDA = 4,      /* CUDA runtime error */
        JCI_ERR_NODEVICE = 5,  /* no CUDA device (no CPU fallback exists) */
        JCI_ERR_IO = 6,        /* file could not be opened / read / written */
        JCI_ERR_FORMAT = 7,    /* malformed SIFS, namelist or vector file */
        JCI_ERR_NOCONV = 8,    /* Davidson hit maxiter; results still valid */
        JCI_ERR_LINALG = 9,    /* subspace eigensolve did not converge */
        JCI_ERR_TIMEOUT = 10,  /* a bounded device wait expired */
        JCI_ERR_BUSY = 11,     /* server admission refused (queue full) */
        JCI_ERR_STATE = 12     /* call out of order (e.g. no integrals set) */
} jci_status;

enum { JCI_FP64 = 0, JCI_FP32 = 1, JCI_MIXED = 2 };

/* Byte layout of the reference's struct occstr (binarystr.h:6-13). */
struct jci_occstr {
        long long byte1;
        int virtx[2];
        int nvrtx;
        int istr[20];
        int yij[20][200];
        int cij[20][200];
};

/* Byte layout of the reference's struct eospace (citruncate.h:9-18). */
struct jci_eospace {
        int docc;
        int actv;
        int virt;
        int nstr;
        int start;
        int pairs[20];
        int npairs;
};

const char *jci_status_string(int status);
/* Number of visible CUDA devices (0 when the driver has none). */
int jci_device_count(void);

/* ---------------------------------------------------------------------
 * Drop-in solve.  Same arguments and meaning as the reference's
 *   int pdavidson(struct occstr *pstrings, struct eospace *peospace,
 *                 int pegrps, struct occstr *qstrings,
 *                 struct eospace *qeospace, int qegrps,
 *                 int **pq_space_pairs, int num_pq, double *moints1,
 *                 double *moints2, int aelec, int belec, int intorb,
 *                 int ndets, double nucrep_e, double frzcore_e,
 *                 int printlvl, int maxiter, int krymin, int krymax,
 *                 int nroots, int prediagr, int refdim, double restol,
 *                 int ga_buffer_len, int nmos, int ndocc, int nactv)
 * (mpi_source/include/pdavidson.h:9, called at execute_pjayci.c:217).
 * The strings, groups and pairs are the ones citrunc produced; only their
 * istr/nvrtx fields and the group table are read.  Files "civec" (and
 * "ci.restart", "hvvec" when not converged) are written to the current
 * directory in the reference's format (mpi_utilities.c:353).  ga_buffer_len
 * is accepted and ignored (the reference overrides it too,
 * pdavidson.c:1327-1335).  Returns 0 on success, a jci_status otherwise.
 * --------------------------------------------------------------------- */
int jci_pdavidson(struct jci_occstr *pstrings, struct jci_eospace *peospace,
                  int pegrps, struct jci_occstr *qstrings,
                  struct jci_eospace *qeospace, int qegrps,
                  int **pq_space_pairs, int num_pq, double *moints1,
                  double *moints2, int aelec, int belec, int intorb,
                  int ndets, double nucrep_e, double frzcore_e, int printlvl,
                  int maxiter, int krymin, int krymax, int nroots,
                  int prediagr, int refdim, double restol, int ga_buffer_len,
                  int nmos, int ndocc, int nactv);

/* ---------------------------------------------------------------------
 * String space handle.
 * --------------------------------------------------------------------- */
typedef struct jci_space jci_space;

/* Build the truncated alpha/beta string space, replacing citrunc
 * (citruncate.c:55, citruncate.h:74) with the electron/orbital counts of
 * the &general namelist.  Limits are the reference's
 * (execute_pjayci.c:96-153): ci alpha/beta electrons <= 20, CI orbitals
 * <= 200, ndocc + nactv <= 64. */
jci_status jci_space_create(int electrons, int orbitals, int nfrzc,
                            int ndocc, int nactv, int nfrzv, int xlvl,
                            jci_space **out);
void jci_space_destroy(jci_space *s);

/* out[10] = {ci_aelec, ci_belec, ci_orbs, nastr, nbstr, pegrps, qegrps,
 *            num_pq, ndets, intorb} (execute_pjayci.c:157-170). */
jci_status jci_space_sizes(const jci_space *s, long long *out);
/* Sorted orbital lists, nstr x nelec, in the order of
 * generate_string_list (citruncate.c:3971). */
jci_status jci_space_strings(const jci_space *s, int spin, int *istr);
/* Per group [docc, actv, virt, nstr, start] (allocate_eospace_array,
 * citruncate.c:121, counts filled by generate_string_list). */
jci_status jci_space_eospaces(const jci_space *s, int spin, int *out);
/* Valid (p,q) group pairs, num_pq x 2 (compute_detnum, citruncate.c:414). */
jci_status jci_space_pq(const jci_space *s, int *out);
/* Address of a sorted orbital list, or -1 (occstr2address,
 * citruncate.c:4093; str_adrfind, straddress.c:48). */
jci_status jci_space_string_index(const jci_space *s, int spin,
                                  const int *orbs, int *index);
/* Single (nrep=1) / double (nrep=2) replacements of string istr landing in
 * group teosp (generate_single_excitations / generate_double_excitations,
 * citruncate.c:755,799).  Entries [index, io0, io1, fo0, fo1, permx];
 * *count receives the number written (out must hold the maximum). */
jci_status jci_space_excitations(const jci_space *s, int spin, int nrep,
                                 int istr, int teosp, int *out, int *count);

/* Upload integrals for this space (packed as moindex.c; norb = CI
 * orbitals) and the core energies (readmointegrals, ioutil.c:416).
 * Builds the integral-dependent device tables. */
jci_status jci_set_integrals(jci_space *s, const double *moints1,
                             const double *moints2, int norb, double nucrep,
                             double frzcore);

/* <i|H|i> for every determinant into host memory
 * (compute_diagonal_iHi, pdavidson.c:1586). */
jci_status jci_hdiag(jci_space *s, double *out);

/* sigma = H v for nvec host vectors (vector-major, ndets each), replacing
 * perform_hvispacefast / compute_hv_newvectorfaster (pdavidson.c:4328,
 * 1778) including the diagonal term (compute_hvc_diagonal_ga, :2105).
 * precision: JCI_FP64 or JCI_FP32 (FP32 storage and accumulation). */
jci_status jci_sigma(jci_space *s, int nvec, const double *v, double *sigma,
                     int precision);

/* Same on device memory: nvec vectors with leading dimension ld (>= ndets,
 * elements); element type double for JCI_FP64, float for JCI_FP32.  The
 * work is queued on `stream` (a cudaStream_t).  NULL = the handle's own
 * stream, ordered after the work already queued on the legacy default
 * stream, which in turn waits for the sigma before its later work. */
jci_status jci_sigma_device(jci_space *s, int nvec, const void *v,
                            void *sigma, long long ld, int precision,
                            void *stream);

/* sigma = H v for ONE device vector (ld = ndets) that allocates no device
 * memory, for callers that cannot call cudaMalloc while they run sigma
 * (a driver capturing its iteration into a CUDA graph, a process under a
 * fixed device-memory budget, an application whose allocator forbids
 * cudaMalloc / cudaFree after start-up).  The alpha-singles product kernel
 * keeps its per-CTA panels in a fixed device array of 64 MiB that lives in
 * the library (every GPU that loads libjci holds it until exit) instead of
 * a buffer allocated on first use; jci_set_integrals must have been called
 * before (it builds the tables this call reads).  Returns JCI_ERR_SPACE,
 * before launching anything, for any space outside these limits:
 *   - one occupation group per spin (FCI / CAS / DOCC+ACTV with xlevel 0);
 *   - n(n+1)/2 + 1 <= 144 for n CI orbitals (n <= 16), the product
 *     kernel's row tile;
 *   - the product kernel's shared memory, Nsingles_alpha x (16 TM + 128)
 *     elements with TM = ceil((n(n+1)/2 + 1) / 16), fits the device's
 *     opt-in limit;
 *   - one alpha row's panel, (n(n+1)/2 + 1) x Nbeta rounded up to 64
 *     elements, fits in 64 MiB;
 *   - the row kernel holds one beta row in shared memory and at most 32
 *     columns per thread (Nbeta <= 16384).
 * The call makes the space's device current.  The first call on a device
 * looks up the array's device address (once per device, made current for
 * the lookup); make that first call before any stream capture.  All calls
 * share the array: calls that overlap on the GPU (other
 * streams, other host threads, other handles on the same device) race and
 * must be serialised by the caller.  Nothing in the array needs clearing: a
 * call writes every panel element before reading it.  No counterpart in the
 * reference (which has no device code). */
jci_status jci_sigma_device_noalloc(jci_space *s, const void *v, void *sigma,
                                    int precision, void *stream);

/* Plan the sigma autotuner picked for this space: mode (0 staged rows;
 * 1, 2, 5 a row kernel followed by the dense product through a global
 * scratch panel (1), consumed chunk by chunk from shared memory (2), or
 * fused with the gather over per-chunk entry lists (5); 3, 4 row streams
 * on C and its transpose followed by the product of mode 1 (3) or of mode
 * 5 (4); 6, 7 the same-spin doubles over groups of 16 consecutive strings,
 * the beta singles as a row stream on the transpose, then the product of
 * mode 1 (6) or of mode 5 (7)), threads per CTA of the row kernel (modes
 * 3-4: of the alpha pass; modes 6-7: of the beta-singles stream, or 0 for
 * the beta singles as products over (N-1)-electron hole strings), `rows`
 * (mode 0: alpha rows staged per pass; modes 1-3 and 6: product CTAs per
 * SM, 0 = as many as fit, plus 16 for the panel cut into 256-column blocks
 * gathered block by block, plus 32 for one panel per alpha row built and
 * gathered by all CTAs from a shared work queue, plus 64 for the per-CTA
 * panel stored compact (only the entries its gather reads) (modes 1, 3,
 * 6); modes 4,
 * 5, 7: column threads of the fused
 * product, 8 (CUDA cores, 32-column chunks) or 16 (tensor cores, 64-column
 * chunks: FP64 mma.sync in FP64, 3xTF32 in FP32), or in FP32 32 / 64 (the
 * tcgen05 engine, 32- / 64-column chunks)), `batch` (modes 1, 2, 5: alpha strings per CTA of the
 * row kernel; modes 3-4: threads per CTA of the beta pass; modes 6-7: the
 * group kernel variant, 1 or 2 columns per thread, or 3, 4: the group's
 * excitation targets split over 4 warps with 2 or 1 columns per lane, or
 * 5-7: the same-spin doubles as dense products over (N-2)-electron hole
 * strings, in the widest column blocks whose scratch fits 1 GiB (5) or
 * 4 GiB (7), or in 64-column blocks (6)), and
 * its timed cost in
 * ms per vector.  All 0 before the first sigma call and on the
 * multi-group path.  No reference counterpart (the reference has no device
 * tuning). */
jci_status jci_sigma_tuning(const jci_space *s, int precision, int *mode,
                            int *threads, int *rows, int *batch, float *ms);

/* Fix the sigma plan instead of autotuning (for tests and measurements),
 * with the mode and arguments as jci_sigma_tuning reports them; threads =
 * 128/256/512/1024 per CTA.  Only for one-group (FCI/CAS) spaces after
 * jci_set_integrals; JCI_ERR_ARG for a plan the space cannot run.  No
 * reference counterpart. */
jci_status jci_sigma_set_plan(jci_space *s, int precision, int mode,
                              int threads, int rows, int batch);

/* Test hook for the device-side wait bounds.  The next sigma whose product
 * runs through the row panels shared by all CTAs (plan rows >= 32) leaves
 * the panel work of its first two alpha rows undone, so the gathers that
 * depend on it wait until their bound (about one second) expires; that
 * sigma's output is then incomplete and the next host-synchronising call
 * (jci_sigma, jci_davidson) returns JCI_ERR_TIMEOUT, after which the space
 * works as before.  JCI_ERR_STATE for a space without device tables.  No
 * reference counterpart. */
jci_status jci_test_expire_next_wait(jci_space *s);

typedef struct {
        int maxiter;      /* &dalginfo defaults: 20 */
        int krymin;       /* 3 */
        int krymax;       /* 8 */
        int nroots;       /* 1 */
        int prediagr;     /* 1 = H over the first refdim dets, 2 = unit
                           * vectors, 3 = start vectors (init or ci.restart) */
        int refdim;       /* 3 */
        double restol;    /* 1e-5 */
        int precision;    /* JCI_FP64 or JCI_MIXED */
        double switch_tol;/* mixed: FP32 sigma until ||r|| < switch_tol */
        int printlvl;
        int write_files;  /* write civec / ci.restart / hvvec to cwd */
        int block;        /* 0 = the reference's root-sequential Davidson;
                           * 1 = block Davidson over all unconverged roots */
        const double *init; /* prediagr == 3: krymin start vectors, or NULL
                             * to read "ci.restart" from the cwd */
        int host_loop;    /* 0 (default): the iterations of the
                           * root-sequential schedule run as a captured CUDA
                           * graph launched in batches, with the control
                           * state on the device; 1: every kernel of every
                           * iteration is launched from the host (same
                           * arithmetic, same results) */
} jci_davidson_opts;

typedef struct {
        int iterations;       /* vectors added (the reference's citer) */
        int sigma_calls;
        long long sigma_vectors;
        double sigma_seconds; /* device time in sigma kernels */
        double total_seconds;
        int converged;
        double rnorm;         /* last residual norm */
        int fp32_sigma_vectors;
} jci_davidson_stats;

/* Fill opts with the &dalginfo defaults (readnamelist.f90:85-92). */
void jci_davidson_defaults(jci_davidson_opts *o);

/* Davidson solve for the lowest nroots (pdavidson.c:39).  energies[nroots]
 * include nucrep + frzcore; civec (nullable) receives nroots x ndets.
 * Returns JCI_ERR_NOCONV when maxiter was reached (outputs still set). */
jci_status jci_davidson(jci_space *s, const jci_davidson_opts *o,
                        double *energies, double *civec,
                        jci_davidson_stats *stats);

/* ---------------------------------------------------------------------
 * Serving: many CI solves of uneven size on one GPU with continuous
 * batching.  Worker slots take queued requests as soon as a slot and HBM
 * budget are free; solves in different slots run concurrently on their own
 * streams, so their kernels overlap on the device.  String spaces (device
 * tables and tuned sigma plans) are cached by their &general values and
 * reused for later requests on the same space (geometry scans).  No
 * counterpart in the reference (one solve per pjayci run).
 * --------------------------------------------------------------------- */
#define JCI_MAX_ROOTS 16

typedef struct jci_server jci_server;

typedef struct {
        int electrons, orbitals, nfrozen, ndocc, nactive, nfrzvirt, xlevel;
        const double *moints1; /* copied by jci_server_submit */
        const double *moints2;
        double nucrep, frzcore;
        int nroots, krymin, krymax, maxiter, refdim;
        double restol;
        int precision;         /* JCI_FP64 or JCI_MIXED */
        double switch_tol;
        int block;             /* 1 = block Davidson */
        long long warm_from;   /* ticket of an earlier, unreleased request on
                                * the same space whose Ritz vectors start
                                * this solve (the request waits for it), or
                                * -1 */
} jci_request;

typedef struct {
        int status;            /* jci_status of the solve */
        int converged;
        int nroots;
        double energies[JCI_MAX_ROOTS];
        int iterations;
        int warm_started;
        long long ndets;
        double queue_seconds;  /* submit -> start */
        double solve_seconds;  /* start -> finish */
        long long sigma_vectors;
        double sigma_seconds;  /* device time in sigma kernels */
} jci_result;

/* hbm_budget_bytes bounds the estimated device memory of the solves running
 * at once (0 = 80 % of free device memory); slots = solves in flight. */
jci_status jci_server_create(size_t hbm_budget_bytes, int slots,
                             jci_server **out);
/* Queue a request; returns JCI_ERR_BUSY if its estimated footprint exceeds
 * the whole budget, JCI_ERR_SPACE / JCI_ERR_ARG for invalid requests. */
jci_status jci_server_submit(jci_server *srv, const jci_request *req,
                             long long *ticket);
/* Wait up to timeout_s (< 0: forever) for a result; JCI_ERR_TIMEOUT if it
 * is not done yet. */
jci_status jci_server_wait(jci_server *srv, long long ticket,
                           double timeout_s, jci_result *out);
/* Result vectors of a finished request (nroots x ndets). */
jci_status jci_server_vectors(jci_server *srv, long long ticket,
                              double *civec);
/* Drop a finished request's stored vectors and result. */
jci_status jci_server_release(jci_server *srv, long long ticket);
/* Finish the queued and running solves, then stop the workers. */
void jci_server_destroy(jci_server *srv);

/* ---------------------------------------------------------------------
 * Input / output formats.
 * --------------------------------------------------------------------- */

/* &general namelist (readnamelist.f90:43-44). */
typedef struct {
        int electrons, orbitals, nfrozen, ndocc, nactive, xlevel, nfrzvirt;
        int printlvl, printwvf;
} jci_general;

/* &dalginfo namelist (readnamelist.f90:45-46, defaults :85-92). */
typedef struct {
        int maxiter, krymin, krymax, nroots, prediagr, refdim, buflen;
        double restol;
} jci_dalginfo;

/* &gpuinfo namelist (new; absent blocks keep the defaults):
 * precision (0 fp64, 2 mixed), switchtol, block (0/1), exactrestol.
 * With exactrestol = 0 (default) restol is rounded as the reference's
 * f10.5 round trip does (readnamelist.f90:105, ioutil.c:337). */
typedef struct {
        int precision;
        double switch_tol;
        int block;
        int exact_restol;
} jci_gpuinfo;

/* Read jayci.in-style namelists (readgeninput / readdaiinput,
 * ioutil.c:313,367).  Any of the output pointers may be NULL. */
jci_status jci_read_namelists(const char *path, jci_general *g,
                              jci_dalginfo *d, jci_gpuinfo *u);

/* Read a SIFS integral file (readmoints.f90:21 with colib sifrsh/sifd2):
 * moints1 (m1cap doubles) and moints2 (m2cap doubles) are zeroed and
 * filled in index1e/index2e packing; *nbft receives the orbital count,
 * *nucrep energy(1) of header 2, *frzcore the H1 core energy.  fsplit 1
 * and 2 (below) are both read. */
jci_status jci_read_moints(const char *path, double *moints1, long long m1cap,
                           double *moints2, long long m2cap, int *nbft,
                           double *nucrep, double *frzcore);

/* Files with fsplit = 2 (info(1) of header 2) keep their 2-e records on a
 * second file, opened by colib's sifo2f (colib8.f:1720) as a plain
 * sequential file of l2rec-word records; the reference's reader refuses
 * them (readmoints.f90:278-282).  jci_read_moints takes them with the 2-e
 * file named path + "2" (moints / moints2, as colib's callers pair
 * aoints / aoints2); jci_read_moints_split names the 2-e file itself (it
 * is only opened when the header says fsplit = 2). */
jci_status jci_read_moints_split(const char *path, const char *path2,
                                 double *moints1, long long m1cap,
                                 double *moints2, long long m2cap, int *nbft,
                                 double *nucrep, double *frzcore);

/* Write a single-symmetry SIFS file with the given packed integrals
 * (colib sifwh / sifew1 / sifew2 layout, 8-bit labels, fsplit = 1). */
jci_status jci_write_moints(const char *path, int nbft,
                            const double *moints1, const double *moints2,
                            double nucrep, double frzcore);
/* The same with fsplit = 2: headers and 1-e records on path, the 2-e
 * records on path2 (sifew2 through colib's aiwrit, colib2.f:178). */
jci_status jci_write_moints_split(const char *path, const char *path2,
                                  int nbft, const double *moints1,
                                  const double *moints2, double nucrep,
                                  double frzcore);

/* Unformatted vector files "civec" / "ci.restart" / "hvvec":
 * int32 dim, int32 len, dim*len float64 (mpi_utilities.c:353,430). */
jci_status jci_write_vectors(const char *path, int dim, int len,
                             const double *v);
jci_status jci_read_vectors(const char *path, int dim, int len, double *v);

/* ---------------------------------------------------------------------
 * Dyson orbitals between an (N+1)-electron and an N-electron CI
 * wavefunction on the same orbitals (the pdycicalc program:
 * run_pdycicalc.c:26, dysoncomp.c:103,220).
 * --------------------------------------------------------------------- */

/* &wavefcn0 / &wavefcn1 namelists of dycicalc.in (readnamelist.f90:47-50,
 * defaults 0 as at :110-158). */
typedef struct {
        int electrons, orbitals, nfrozen, ndocc, nactive, nfrzvirt, xlevel;
        int nstates;
} jci_wavefcn;

/* Read dycicalc.in (readwf0input / readwf1input / readdysoninput,
 * ioutil.c:154-260): &wavefcn0 (N+1 electrons), &wavefcn1 (N electrons)
 * and &dysonorbital states0 / states1 (five 1-based states each, default
 * states0 = states1 = 1).  *nst0 / *nst1 receive the position of the last
 * nonzero entry, as the reference counts them; states arrays hold 5. */
jci_status jci_read_dycicalc(const char *path, jci_wavefcn *wf0,
                             jci_wavefcn *wf1, int *states0, int *nst0,
                             int *states1, int *nst1);

/* Dyson orbitals (compute_dyson_orbital_a / _b and the sqrt(N+1)
 * prefactor, run_pdycicalc.c:376-414).  s0 is the (N+1)-electron space,
 * s1 the N-electron space (electrons one fewer, same orbitals, frozen,
 * DOCC, active and frozen-virtual counts: check_wavefunction_input,
 * run_pdycicalc.c:458).  v0 holds nstates0 x ndets(s0) and v1 nstates1 x
 * ndets(s1) host vectors, state-major.  For every determinant of s0 and
 * every electron of the spin whose count differs (beta when the N+1
 * electron count is even, else alpha), the electron is removed; when the
 * string and determinant exist in s1 the product
 * v0[states0[j]] v1[states1[k]] is added to that orbital of Dyson orbital
 * j*nst1 + k (no phase factor, as the reference).  dyorb receives
 * (nst0*nst1) x orbitals values (orbitals of &wavefcn0, indexed by CI
 * orbital number - 1).  Runs on the device; deterministic summation. */
jci_status jci_dyson(jci_space *s0, jci_space *s1, const double *v0,
                     int nstates0, const double *v1, int nstates1,
                     const int *states0, int nst0, const int *states1,
                     int nst1, double *dyorb);

/* Write dysonorb.dat in the format of print_dysonorbitals_to_file
 * (run_pdycicalc.c:674-712). */
jci_status jci_write_dysonorb(const char *path, int ndyorbs, int orbs,
                              const double *dyorb, const int *states0,
                              int nst0, const int *states1, int nst1);

#ifdef __cplusplus
}
#endif
#endif
