"""The hole-string forms of the same-spin excitations (no GPU needed).

jci_fci_pairs.cu evaluates the same-spin doubles through (N-2)-electron hole
strings K: for I = K + {i,j} and J = K + {k,l} with {i,j} and {k,l}
disjoint,
    <I|H|J> = phi(K;i,j) phi(K;k,l) [(ik|jl) - (il|jk)],
    phi(K;k,l) = (-1)^(#K below k + #K below l),
and the singles through (N-1)-electron hole strings K: for I = K + k and
J = K + l the element's phase is phi(K;k) phi(K;l), phi(K;x) = (-1)^(#K
below x), and its one-body part depends on K and (k,l) only.  These tests
check both rules element by element against the oracle's Hamiltonian (the
restatement of hmatels_2xaa and hmatels_1x, mpi_source/action_util.c:210,
237-245), on CAS(7e,7o) with alpha excitations at a fixed beta string.
"""
import itertools

import numpy as np
import pytest

from jayci_b200.synth import make_integrals, unpack_integrals
from oracle.oracle import OracleSpace

N_ORB, N_EL = 7, 3  # orbitals, electrons per spin


@pytest.fixture(scope="module")
def hamiltonian():
    ints = make_integrals(N_ORB, N_ORB, 5)
    m1, m2 = ints.packed()
    h, eri = unpack_integrals(m1, m2, N_ORB)
    o = OracleSpace(N_EL, N_EL, N_ORB)
    sa = [tuple(int(x) for x in s) for s in o.strings(0)]
    sb = [tuple(int(x) for x in s) for s in o.strings(1)]
    H = o.sigma(m1, m2, np.eye(o.ndets))
    return h, eri, sa, sb, H


def _below(K, x):
    return sum(1 for y in K if y < x)


def test_same_spin_doubles_through_hole_pairs(hamiltonian):
    h, eri, sa, sb, H = hamiltonian
    ia = {s: i for i, s in enumerate(sa)}
    nb = len(sb)
    R = np.zeros((len(sa), len(sa)))
    seen = np.zeros_like(R, dtype=int)
    for K in itertools.combinations(range(1, N_ORB + 1), N_EL - 2):
        free = [x for x in range(1, N_ORB + 1) if x not in K]
        pairs = list(itertools.combinations(free, 2))
        for (i, j) in pairs:
            I = ia[tuple(sorted(K + (i, j)))]
            for (k, l) in pairs:
                if {i, j} & {k, l}:
                    continue
                J = ia[tuple(sorted(K + (k, l)))]
                phase = (-1) ** (_below(K, i) + _below(K, j) + _below(K, k) + _below(K, l))
                R[I, J] += phase * (eri[i - 1, k - 1, j - 1, l - 1] -
                                    eri[i - 1, l - 1, j - 1, k - 1])
                seen[I, J] += 1
    checked = 0
    for I in range(len(sa)):
        for J in range(len(sa)):
            double = len(set(sa[I]) - set(sa[J])) == 2
            # every double has exactly one hole string, nothing else has one
            assert seen[I, J] == (1 if double else 0)
            if not double:
                continue
            for b in range(nb):
                assert abs(H[I * nb + b, J * nb + b] - R[I, J]) <= 1e-12
                checked += 1
    assert checked > 0


def test_same_spin_singles_through_hole_strings(hamiltonian):
    h, eri, sa, sb, H = hamiltonian
    ia = {s: i for i, s in enumerate(sa)}
    nb = len(sb)
    checked = 0
    for K in itertools.combinations(range(1, N_ORB + 1), N_EL - 1):
        free = [x for x in range(1, N_ORB + 1) if x not in K]
        for k, l in itertools.permutations(free, 2):
            I = ia[tuple(sorted(K + (k,)))]
            J = ia[tuple(sorted(K + (l,)))]
            phase = (-1) ** (_below(K, k) + _below(K, l))
            # one-body part: depends on K and (k, l) only
            a1 = h[k - 1, l - 1] + sum(eri[k - 1, l - 1, m - 1, m - 1] -
                                       eri[k - 1, m - 1, m - 1, l - 1] for m in K)
            for b, sbeta in enumerate(sb):
                coul = sum(eri[k - 1, l - 1, m - 1, m - 1] for m in sbeta)
                assert abs(H[I * nb + b, J * nb + b] - phase * (a1 + coul)) <= 1e-12
                checked += 1
    assert checked > 0
