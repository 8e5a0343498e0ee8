"""The gathers' launch variants: the copy-engine streamed ones (4, 5) sum
every row and column in the same order as the register-streamed ones with
the same lanes per row (0 and 3), and the two 16-lane ones (6, 7) agree with
each other, so a resident run gives bit-identical results in both
precisions; a pinned choice repeats a run bit for bit."""
import numpy as np
import pytest

from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu

FIELDS = (_lib.F_DSP_TOT, _lib.F_VEL, _lib.F_ACL, _lib.F_STRESS, _lib.F_EPS, _lib.F_FINT)


def _run(case, mode, variants, steps=40):
    m = mega.Mega(case, _lib.params(**cases.param_kwargs(case)))
    m.search_and_shapes()
    m.set_variants(*variants, mode=mode)
    m.step(steps, 3.9e-8, mode=mode)
    out = {f: m.download(f) for f in FIELDS}
    s = m.scalars()
    m.close()
    return out, s


@pytest.mark.parametrize("mode", ["mixed", "fp64"])
@pytest.mark.parametrize("pair", [((0, 0), (4, 4)), ((3, 3), (5, 5)), ((0, 4), (4, 0)), ((6, 6), (7, 7))])
def test_streamed_variants_are_bit_identical(bar16k, mode, pair):
    a, sa = _run(bar16k, mode, pair[0])
    b, sb = _run(bar16k, mode, pair[1])
    for f in FIELDS:
        np.testing.assert_array_equal(a[f], b[f])
    # the energy is a sum of per-block atomics, whose order the scheduler picks
    assert abs(sa["kin_energy"] - sb["kin_energy"]) <= 1e-13 * abs(sa["kin_energy"])


def test_repeat_run_is_bit_identical(bar16k):
    a, _ = _run(bar16k, "mixed", (4, 4), steps=60)
    b, _ = _run(bar16k, "mixed", (4, 4), steps=60)
    for f in FIELDS:
        np.testing.assert_array_equal(a[f], b[f])


def test_set_variants_arguments(bar16k):
    m = mega.Mega(bar16k, _lib.params(**cases.param_kwargs(bar16k)))
    with pytest.raises(_lib.MegaError):
        m.set_variants(0, 0)          # before the search
    m.search_and_shapes()
    with pytest.raises(_lib.MegaError):
        m.set_variants(8, 0)          # no such variant
    m.close()
