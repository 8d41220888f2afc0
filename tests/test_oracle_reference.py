"""The CPU oracle against the reference library itself, bit for bit.

Runs only where the reference was built from its sources into oracle/_ref
(make -C oracle ref). Precisions DEFAULT, F32F32_ACCUM_F32 and
F64F64_ACCUM_F64 are checked against the default build; F16F16_ACCUM_F16,
F16F16_ACCUM_F32 and binary16 storage against the build with
TAPP_REFERENCE_ENABLE_F16. (BF16BF16_ACCUM_F32 has no reference: the
reference's BF16 build does not compile.)
"""
import itertools

import numpy as np
import pytest

from families import family_cases, random_case

oracle_mod = pytest.importorskip("oracle")
REF = oracle_mod.reference_lib()
REF16 = oracle_mod.reference_lib(f16=True)
pytestmark = pytest.mark.skipif(REF is None or REF16 is None, reason="reference not built (make -C oracle ref)")


def _same(case, lib, oracle):
    c1, c2 = case.copy(), case.copy()
    e1 = c1.run(lib)
    e2 = oracle.execute(c2)
    assert e1 == e2
    assert np.array_equal(c1.D.buf.view(np.uint8), c2.D.buf.view(np.uint8)), case.name


@pytest.mark.parametrize("prec", [-1, 0, 1])
def test_families_bit_exact(oracle, prec):
    for fam, case in family_cases(1000 + prec, 3):
        case.prec = prec
        _same(case, REF, oracle)


@pytest.mark.parametrize("prec", [-1, 0, 1])
def test_mixed_storage_types_bit_exact(oracle, prec):
    rng = np.random.default_rng(77 + prec)
    for types in itertools.product((0, 1, 2, 3), repeat=4):
        if prec != -1 and types[0] in (0, 1) and types[1] in (2, 3):
            continue  # reference leaves B's imaginary sum uninitialised there (product.c:381)
        case = random_case(rng, types=types, prec=prec, n_isoA=int(rng.integers(0, 2)),
                           n_isoB=int(rng.integers(0, 2)), n_repA=int(rng.integers(0, 2)),
                           subtensor=True, mixed=True)
        _same(case, REF, oracle)


@pytest.mark.parametrize("prec", [4, 5])
def test_half_precisions_bit_exact(oracle, prec):
    rng = np.random.default_rng(300 + prec)
    for types in [(0, 0, 0, 0), (1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3), (4, 4, 4, 4), (4, 0, 4, 0), (0, 4, 0, 4)]:
        for i in range(4):
            case = random_case(rng, types=types, prec=prec, n_isoA=i % 2, n_repA=(i // 2) % 2,
                               mixed=(i == 3), subtensor=True)
            _same(case, REF16, oracle)


def test_binary16_storage_default_precision(oracle):
    rng = np.random.default_rng(11)
    for i in range(12):
        case = random_case(rng, types=(4, 4, 4, 4), prec=-1, n_isoA=i % 2, subtensor=True)
        _same(case, REF16, oracle)
