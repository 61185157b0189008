"""Seeded synthetic molecular-orbital integrals for the CI workloads.

There is no public benchmark suite for this path, so every workload is a
seeded synthetic integral set with the shapes and value distributions of a
small molecule's MO integrals:

* orbital energies eps_p evenly spaced in [-2, +1] Eh,
* h_pq = eps_p delta_pq + S_pq with S = (A + A^T)/sqrt(2), A_ij ~ N(0, 0.05^2),
* a rank-R symmetric factorisation (pq|rs) = sum_K L^K_pq L^K_rs with
  L^K = (G^K + G^K^T)/sqrt(2), G^K_ij ~ N(0, 1), rescaled
  L^K_pq <- s_p s_q L^K_pq with s_p = (t_p / D_p)^(1/4),
  D_p = sum_K (L^K_pp)^2 and t_p ~ U[0.5, 1.0], so that (pp|pp) = t_p exactly
  and the two-electron tensor stays positive semi-definite (8-fold symmetric),
* E_nuc = 10.0 Eh.

Random draws come from ``numpy.random.default_rng(seed)`` (PCG64) in the
order A, G, t.

A frozen core is folded the way a quantum-chemistry front end hands it to the
CI code (the reference never folds it itself; it reads the folded one-electron
matrix and the core energy from the SIFS H1 record, readmoints.f90:164-169):
h'_pq = h_pq + sum_c [2 (pq|cc) - (pc|cq)] and
E_fc = 2 sum_c h_cc + sum_{c,c'} [2 (cc|c'c') - (cc'|c'c)].

Packing follows the reference's moindex.c:14-41: one-electron values at
index1e(i, j) - 1 (1-based lower triangle), two-electron values at
index2e(i, j, k, l) - 1 = index1e(index1e(i, j), index1e(k, l)) - 1.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

E_NUC = 10.0


def index1e(i, j):
    """1-based lower-triangle index (moindex.c:14)."""
    i = np.asarray(i)
    j = np.asarray(j)
    hi = np.maximum(i, j)
    lo = np.minimum(i, j)
    return hi * (hi - 1) // 2 + lo


def index2e(i, j, k, l):
    """1-based packed two-electron index (moindex.c:30)."""
    return index1e(index1e(i, j), index1e(k, l))


@dataclass
class Integrals:
    """Dense MO integrals over the CI orbitals plus core energies."""

    h: np.ndarray          # (n, n) one-electron matrix (frozen core folded in)
    eri: np.ndarray        # (n, n, n, n) chemists' notation (pq|rs)
    e_nuc: float
    e_fc: float            # frozen-core energy (0.0 without frozen core)

    @property
    def norb(self) -> int:
        return self.h.shape[0]

    def packed(self):
        """(moints1, moints2) in the reference's 1-based packed layout."""
        return pack_integrals(self.h, self.eri)


def pack_integrals(h: np.ndarray, eri: np.ndarray):
    n = h.shape[0]
    m1len = n * (n + 1) // 2
    m2len = m1len * (m1len + 1) // 2
    m1 = np.zeros(m1len)
    m2 = np.zeros(m2len)
    idx = np.arange(1, n + 1)
    I, J = np.meshgrid(idx, idx, indexing="ij")
    mask = I >= J
    m1[index1e(I[mask], J[mask]) - 1] = h[I[mask] - 1, J[mask] - 1]
    pair_i, pair_j = I[mask], J[mask]                       # pairs with i >= j
    ij = index1e(pair_i, pair_j)
    P, Q = np.meshgrid(np.arange(len(ij)), np.arange(len(ij)), indexing="ij")
    keep = ij[P] >= ij[Q]
    P, Q = P[keep], Q[keep]
    m2[index1e(ij[P], ij[Q]) - 1] = eri[pair_i[P] - 1, pair_j[P] - 1,
                                        pair_i[Q] - 1, pair_j[Q] - 1]
    return m1, m2


def unpack_integrals(m1: np.ndarray, m2: np.ndarray, n: int):
    idx = np.arange(1, n + 1)
    I, J = np.meshgrid(idx, idx, indexing="ij")
    h = m1[index1e(I, J) - 1]
    P, Q, R, S = np.meshgrid(idx, idx, idx, idx, indexing="ij")
    eri = m2[index2e(P, Q, R, S) - 1]
    return h, eri


def _raw(n: int, rank: int, seed: int, eps: np.ndarray):
    rng = np.random.default_rng(seed)
    a = rng.normal(0.0, 0.05, size=(n, n))
    h = np.diag(eps) + (a + a.T) / np.sqrt(2.0)
    g = rng.standard_normal(size=(rank, n, n))
    L = (g + np.transpose(g, (0, 2, 1))) / np.sqrt(2.0)
    t = rng.uniform(0.5, 1.0, size=n)
    d = np.sum(L[:, np.arange(n), np.arange(n)] ** 2, axis=0)
    s = (t / d) ** 0.25
    L = L * s[None, :, None] * s[None, None, :]
    eri = np.einsum("kpq,krs->pqrs", L, L)
    return h, eri


def make_integrals(n: int, rank: int, seed: int, nfrozen: int = 0,
                   core_eps=(-20.0, -19.5)) -> Integrals:
    """Seeded integrals over n CI orbitals (after folding nfrozen cores).

    With nfrozen > 0, n + nfrozen orbitals are generated: the nfrozen core
    orbitals first, with energies ``core_eps``, then n orbitals evenly spaced
    in [-2, +1] Eh; the core is folded into h and E_fc.
    """
    ntot = n + nfrozen
    eps = np.concatenate([np.asarray(core_eps[:nfrozen], float),
                          np.linspace(-2.0, 1.0, n)])
    h, eri = _raw(ntot, rank, seed, eps)
    e_fc = 0.0
    if nfrozen:
        c = np.arange(nfrozen)
        a = np.arange(nfrozen, ntot)
        hf = h + 2.0 * np.einsum("pqcc->pq", eri[:, :, c][:, :, :, c]) \
            - np.einsum("pccq->pq", eri[:, c][:, :, c])
        e_fc = 2.0 * np.trace(h[np.ix_(c, c)]) + \
            2.0 * np.einsum("ccdd->", eri[np.ix_(c, c, c, c)]) - \
            np.einsum("cddc->", eri[np.ix_(c, c, c, c)])
        h = hf[np.ix_(a, a)]
        eri = eri[np.ix_(a, a, a, a)]
    return Integrals(h=np.ascontiguousarray(h), eri=np.ascontiguousarray(eri),
                     e_nuc=E_NUC, e_fc=float(e_fc))


def perturb(ints: Integrals, seed: int, sigma: float = 1e-3) -> Integrals:
    """One geometry-scan step: symmetric N(0, sigma^2) perturbations of h and
    of a rank-n factor added to the two-electron tensor (kept 8-fold
    symmetric and PSD-preserving to first order)."""
    rng = np.random.default_rng(seed)
    n = ints.norb
    a = rng.normal(0.0, sigma, size=(n, n))
    h = ints.h + (a + a.T) / np.sqrt(2.0)
    g = rng.normal(0.0, sigma, size=(n, n))
    dl = (g + g.T) / np.sqrt(2.0)
    # (pq|rs) += dl_pq dl_rs keeps every index symmetry and the PSD property
    eri = ints.eri + np.einsum("pq,rs->pqrs", dl, dl)
    return Integrals(h=h, eri=eri, e_nuc=ints.e_nuc, e_fc=ints.e_fc)


# Workloads named by what they are (electrons, orbitals, roots, rank, seed).
WORKLOADS = {
    "cas10_10": dict(n=10, k=5, rank=10, seed=101, nfrozen=0, nroots=1),
    "fci12_12": dict(n=12, k=6, rank=12, seed=102, nfrozen=0, nroots=3),
    "fci14_14_fc2": dict(n=14, k=7, rank=14, seed=103, nfrozen=2, nroots=4),
    "fci16_16": dict(n=16, k=8, rank=16, seed=104, nfrozen=0, nroots=1),
}


def workload_integrals(name: str) -> Integrals:
    w = WORKLOADS[name]
    return make_integrals(w["n"], w["rank"], w["seed"], w["nfrozen"])
