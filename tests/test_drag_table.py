"""The served drag table's coefficient table against the reference's
AeroCoefficientTable (src/atmo/aero_table.cpp:24-83), compiled from the
reference sources into the adapter harness: the same lookups (interpolated
and clamped) and the same refusals."""
import math

import numpy as np
import pytest

from orrery_b200.drag_table import CdTable


def _oracle():
    from oracle import oracle as O
    if not O.adapter_available():
        pytest.skip("adapter harness not built (needs the reference tree at build time)")
    return O


def test_lookup_matches_the_reference_table():
    O = _oracle()
    rng = np.random.default_rng(5)
    for n in (1, 2, 5, 9):
        mach = np.cumsum(rng.uniform(0.05, 1.0, n))
        cd = rng.uniform(0.2, 2.0, n)
        samples = list(zip(mach, cd))
        query = np.concatenate([mach, rng.uniform(0.0, mach[-1] + 1.0, 40), [0.0, mach[0], mach[-1] + 5.0]])
        ref_cd, ref_clamped = O.reference_cd_lookup(samples, query)
        table = CdTable(samples)
        for q, c, cl in zip(query, ref_cd, ref_clamped):
            got = table.lookup(q)
            assert got.cd == c, (q, got.cd, c)
            assert got.clamped == cl, (q, got.clamped, cl)


@pytest.mark.parametrize("samples", [[], [(1.0, 0.0)], [(1.0, 1.0), (1.0, 2.0)], [(2.0, 1.0), (1.0, 2.0)],
                                     [(-1.0, 1.0)], [(1.0, math.inf)]])
def test_refusals_match_the_reference(samples):
    O = _oracle()
    with pytest.raises(O.ReferenceError_) as ref:
        O.reference_cd_lookup(samples, [1.0])
    with pytest.raises(ValueError) as ours:
        CdTable(samples)
    assert str(ours.value) == str(ref.value)
