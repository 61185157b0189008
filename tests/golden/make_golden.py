"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference's own mpi_source C code (oracle/_ref/libjayci_ref.so,
built from the read-only reference tree by ``make -C oracle``) single-rank
and single-threaded on seeded synthetic integrals, and stores what it
produces: string lists, group tables, (p,q) pairs, determinant triples,
yij/cij tables, excitation lists, <i|H|i>, sigma on seeded random vectors,
Davidson energies / vectors, and Dyson orbitals between (N+1)- and
N-electron wavefunctions.

    JAYCI_REF=<reference checkout> OMP_NUM_THREADS=1 python tests/golden/make_golden.py
    python tests/golden/make_golden.py fci12_12 fci14_14_fc2 fci16_16

Only this script touches the reference; the tests read the .npz files.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from jayci_b200.synth import make_integrals  # noqa: E402
from oracle.oracle import RefSpace  # noqa: E402

# name: (&general values, integral rank, seed, davidson options or None)
CASES = {
    # CAS(6,6): 3 alpha / 3 beta electrons in 6 orbitals, 400 determinants
    "cas6_6": (dict(electrons=6, orbitals=6), 6, 11,
               dict(krymin=4, krymax=10, nroots=2, refdim=8)),
    # odd electron count: 4 alpha / 3 beta in 7 orbitals
    "cas7_7": (dict(electrons=7, orbitals=7), 7, 12,
               dict(krymin=3, krymax=8, nroots=1, refdim=6)),
    # truncated: 2 DOCC, 4 ACTV, 2 VIRT, excitation level 2
    "trunc6_8_x2": (dict(electrons=6, orbitals=8, ndocc=2, nactv=4, xlvl=2), 8, 13,
                    dict(krymin=4, krymax=10, nroots=2, refdim=8)),
    # truncated with a frozen core and a frozen virtual, excitation level 1
    "trunc10_12_fc_x1": (dict(electrons=10, orbitals=12, nfrzc=1, ndocc=3, nactv=4,
                              nfrzv=1, xlvl=1), 10, 14,
                         dict(krymin=3, krymax=8, nroots=1, refdim=6)),
    # the 63 504-determinant CAS(10,10) workload (seed 101, rank 10)
    "cas10_10": (dict(electrons=10, orbitals=10), 10, 101,
                 dict(krymin=4, krymax=12, nroots=1, refdim=8)),
}


def make(name):
    gen, rank, seed, dav = CASES[name]
    ref = RefSpace(gen["electrons"], gen["orbitals"], gen.get("nfrzc", 0),
                   gen.get("ndocc", 0), gen.get("nactv"), gen.get("nfrzv", 0),
                   gen.get("xlvl", 0))
    ints = make_integrals(ref.norb, rank, seed)
    m1, m2 = ints.packed()
    out = dict(general=np.array([gen["electrons"], gen["orbitals"], gen.get("nfrzc", 0),
                                 gen.get("ndocc", 0), ref.nactv, gen.get("nfrzv", 0),
                                 gen.get("xlvl", 0)]),
               rank=rank, seed=seed, m1=m1, m2=m2, e_nuc=ints.e_nuc,
               sizes=np.array([ref.na, ref.nb, ref.norb, ref.nastr, ref.nbstr, ref.pegrps,
                               ref.qegrps, ref.npq, ref.ndets]))
    for sp in (0, 1):
        istr, b1, vx, nv = ref.strings(sp)
        out[f"istr{sp}"] = istr
        out[f"byte1_{sp}"] = b1
        out[f"eosp{sp}"] = ref.eospaces(sp)[:, :6]
        if ref.ndets < 100000:
            y, c = ref.yij_cij(sp)
            out[f"yij{sp}"] = y
            out[f"cij{sp}"] = c
        # excitation lists of a few strings into every group
        ns = ref.nastr if sp == 0 else ref.nbstr
        ng = ref.pegrps if sp == 0 else ref.qegrps
        rows = []
        for s in sorted(set([0, 1, ns // 3, ns // 2, ns - 1])):
            for g in range(ng):
                for nrep in (1, 2):
                    for r in ref.excitations(sp, nrep, s, g):
                        rows.append([s, g, nrep] + list(r))
        out[f"exc{sp}"] = np.array(rows, np.int32).reshape(-1, 9)
    out["pq"] = ref.pq()
    out["wlist"] = ref.wlist()
    out["hdiag"] = ref.hdiag(m1, m2)
    rng = np.random.default_rng(seed + 1000)
    V = rng.standard_normal((2, ref.ndets))
    out["sigma_v"] = V
    out["sigma"] = ref.sigma(m1, m2, V)
    if dav:
        civ, _ = ref.davidson(m1, m2, ints.e_nuc, 0.0, maxiter=500, prediagr=1,
                              restol=1e-9, **dav)
        H = None
        # Rayleigh quotients of the reference's result vectors (its energies)
        S = ref.sigma(m1, m2, civ)
        e = np.einsum("ij,ij->i", civ, S) + ints.e_nuc
        out["dav_opts"] = np.array([dav["krymin"], dav["krymax"], dav["nroots"],
                                    dav["refdim"]])
        out["energies"] = e
        out["civec"] = civ
        del H
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, ref.ndets, out.get("energies"))


# Dyson orbitals (run_pdycicalc.c / dysoncomp.c): (N+1) and N electron
# wavefunctions on the same orbitals and integrals, their lowest states from
# the reference's pdavidson, and the reference's Dyson orbitals.
# name: (&wavefcn0, &wavefcn1, nstates0, nstates1, states0, states1, rank, seed)
DYSON_CASES = {
    # anion doublet 7e/6o (alpha electrons compared) -> neutral 6e/6o
    "dyson_cas7_6": ((7, 6, 0, 0, 6, 0, 0), (6, 6, 0, 0, 6, 0, 0), 2, 3, [1], [1, 2], 6, 31),
    # 8e -> 7e (beta electrons compared), DOCC/ACTV/VIRT excitation level 2
    "dyson_trunc8_8_x2": ((8, 8, 0, 2, 4, 0, 2), (7, 8, 0, 2, 4, 0, 2), 2, 2, [1, 2], [1, 2],
                          8, 32),
}


def make_dyson(name):
    from oracle.oracle import ref_dyson
    g0, g1, n0, n1, st0, st1, rank, seed = DYSON_CASES[name]
    ints = make_integrals(g0[1] - g0[2] - g0[5], rank, seed)
    m1, m2 = ints.packed()
    vecs = []
    for g, n in ((g0, n0), (g1, n1)):
        ref = RefSpace(*g)
        civ, _ = ref.davidson(m1, m2, ints.e_nuc, 0.0, maxiter=500, krymin=max(4, n),
                              krymax=12, nroots=n, prediagr=1, refdim=8, restol=1e-9)
        vecs.append(civ)
    dy = ref_dyson(g0, g1, vecs[0], vecs[1], st0, st1)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), general0=np.array(g0),
                        general1=np.array(g1), v0=vecs[0], v1=vecs[1],
                        states0=np.array(st0), states1=np.array(st1), dyorb=dy)
    print(name, vecs[0].shape, vecs[1].shape, np.abs(dy).max())


# Bench-size workloads (jayci_b200.synth.WORKLOADS), written as
# bench_<workload>.npz: full vectors do not fit in the repository, so these
# fixtures hold samples.  Input vectors are the
# counter-hash vectors of seeded.py, which the tests regenerate.
#   fci12_12      the reference's own sigma (full, then sampled) and the
#                 reference's own pdavidson with the bench's &dalginfo
#                 (krymin 6, krymax 24, refdim 12, 3 roots, restol 1e-8);
#   fci14_14_fc2, fci16_16
#                 sigma at sampled rows from the oracle's row gather
#                 (jo_sigma_rows), whose agreement with the reference's own
#                 sigma is pinned on the fci12_12 rows by the CPU tests.
SIGMA_SEED, PROJ_SEEDS, ROW_SEED, NROWS = 1, (1001, 1002, 1003, 1004), 7, 4096
TOPK = 2048


def _projections(x, n):
    from seeded import hash_vector
    return np.array([hash_vector(n, s) @ x for s in PROJ_SEEDS])


def make_large(name, davidson=True):
    from seeded import hash_vector, sample_rows

    from jayci_b200.synth import WORKLOADS, workload_integrals
    from oracle.oracle import OracleSpace
    w = WORKLOADS[name]
    ints = workload_integrals(name)
    m1, m2 = ints.packed()
    n, k = w["n"], w["k"]
    out = dict(general=np.array([2 * k + 2 * w["nfrozen"], n + w["nfrozen"], w["nfrozen"],
                                 0, n, 0, 0]),
               m1_sum=m1.sum(), m2_sum=m2.sum(), e_nuc=ints.e_nuc, e_fc=ints.e_fc,
               sigma_seed=SIGMA_SEED, proj_seeds=np.array(PROJ_SEEDS))
    if name == "fci12_12":
        ref = RefSpace(2 * k, n)
        N = ref.ndets
        v = hash_vector(N, SIGMA_SEED)
        S = ref.sigma(m1, m2, v)[0]
        rows = sample_rows(N, NROWS, ROW_SEED)
        out.update(ndets=N, rows=rows, sigma_rows=S[rows], sigma_norm2=S @ S,
                   sigma_proj=_projections(S, N), source="reference")
        if davidson:
            kmin, kmax, refdim, nroots = 6, 24, 12, 3
            civ, _ = ref.davidson(m1, m2, ints.e_nuc, 0.0, maxiter=500, krymin=kmin,
                                  krymax=kmax, nroots=nroots, prediagr=1, refdim=refdim,
                                  restol=1e-8)
            Sc = ref.sigma(m1, m2, civ)
            e = np.einsum("ij,ij->i", civ, Sc) + ints.e_nuc
            top = np.argsort(-np.abs(civ), axis=1)[:, :TOPK]
            out.update(dav_opts=np.array([kmin, kmax, nroots, refdim]), energies=e,
                       civec_idx=top, civec_val=np.take_along_axis(civ, top, axis=1),
                       civec_proj=np.array([_projections(c, N) for c in civ]),
                       civec_res=np.linalg.norm(Sc - (e - ints.e_nuc)[:, None] * civ, axis=1))
    else:
        o = OracleSpace(k, k, n)
        N = o.ndets
        v = hash_vector(N, SIGMA_SEED)
        rows = sample_rows(N, NROWS, ROW_SEED)
        out.update(ndets=N, rows=rows, sigma_rows=o.sigma_rows(m1, m2, v, rows),
                   source="oracle")
    np.savez_compressed(os.path.join(HERE, f"bench_{name}.npz"), **out)
    print(name, out["ndets"], out.get("energies"))


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    for n in (sys.argv[1:] or list(CASES) + list(DYSON_CASES)):
        if n in DYSON_CASES:
            make_dyson(n)
        elif n in CASES:
            make(n)
        else:
            make_large(n)
