"""The identity behind the ordered warp sums of the water PBF and XSPH passes: adding the
27 cell partials in order equals adding only the partials that are not +0, with one
addition of +0 for each run of +0 partials left out (float32, round to nearest).  Checked
bit for bit on partials rich in +0, -0, infinities, NaN and subnormals."""
import numpy as np
import pytest

F = np.float32


def full_sum(acc, parts):
    for p in parts:
        acc = F(acc + p)
    return acc


def skipping_sum(acc, parts):
    """The kernel's rule, one component: parts[k] is left out when its bits are those of +0."""
    nz = [k for k, p in enumerate(parts) if np.float32(p).view(np.uint32) != 0]
    nxt = 0
    for k in nz:
        if k > nxt:
            acc = F(acc + F(0.0))
        acc = F(acc + parts[k])
        nxt = k + 1
    if nxt < len(parts):
        acc = F(acc + F(0.0))
    return acc


def bits(x):
    return np.float32(x).view(np.uint32)


VALUES = [F(0.0), F(-0.0), F(1.5), F(-2.25), F(np.inf), F(-np.inf), F(1e-45), F(-1e-45), F(3.4e38), F(-3.4e38),
          F(1e-3), F(-1e-3)]


@pytest.mark.parametrize("seed", range(20))
def test_skipping_plus_zero_partials_is_exact(seed):
    rng = np.random.default_rng(seed)
    with np.errstate(all="ignore"):
        for _ in range(400):
            # mostly +0 partials, as in cells without neighbours of a kind
            kinds = rng.integers(0, 4, 27)
            parts = [F(0.0) if k < 2 else VALUES[rng.integers(0, len(VALUES))] if k == 2
                     else F(rng.normal()) for k in kinds]
            acc0 = VALUES[rng.integers(0, len(VALUES))] if rng.random() < 0.5 else F(rng.normal())
            a, b = full_sum(acc0, parts), skipping_sum(acc0, parts)
            if np.isnan(a):
                assert np.isnan(b)
            else:
                assert bits(a) == bits(b), (acc0, parts, a, b)


def test_negative_zero_total_becomes_positive_zero():
    # -0 + (+0) = +0: a run of +0 partials after a -0 total must still turn it into +0
    parts = [F(-0.0), F(0.0), F(0.0)]
    assert bits(full_sum(F(-0.0), parts)) == bits(F(0.0))
    assert bits(skipping_sum(F(-0.0), parts)) == bits(F(0.0))
    # ... a -0 total that meets only -0 partials stays -0
    parts = [F(-0.0), F(-0.0)]
    assert bits(full_sum(F(-0.0), parts)) == bits(F(-0.0))
    assert bits(skipping_sum(F(-0.0), parts)) == bits(F(-0.0))
    # ... and one +0 partial anywhere before the end makes it +0 for good
    parts = [F(0.0), F(-0.0)]
    assert bits(full_sum(F(-0.0), parts)) == bits(F(0.0))
    assert bits(skipping_sum(F(-0.0), parts)) == bits(F(0.0))


def skipping_sum3(acc, parts):
    """The kernel's rule on float3 partials: a partial is left out only when all three of its
    components are +0; a run of left-out partials is one addition of (+0, +0, +0)."""
    nz = [k for k, p in enumerate(parts) if any(bits(c) != 0 for c in p)]
    acc = list(acc)
    nxt = 0
    for k in nz:
        if k > nxt:
            acc = [F(a + F(0.0)) for a in acc]
        acc = [F(a + c) for a, c in zip(acc, parts[k])]
        nxt = k + 1
    if nxt < len(parts):
        acc = [F(a + F(0.0)) for a in acc]
    return acc


@pytest.mark.parametrize("seed", range(10))
def test_float3_rule_matches_componentwise_sums(seed):
    rng = np.random.default_rng(100 + seed)
    with np.errstate(all="ignore"):
        for _ in range(200):
            parts = []
            for _ in range(27):
                if rng.random() < 0.6:
                    parts.append((F(0.0), F(0.0), F(0.0)))
                else:
                    parts.append(tuple(F(0.0) if rng.random() < 0.4 else VALUES[rng.integers(0, len(VALUES))]
                                       if rng.random() < 0.3 else F(rng.normal()) for _ in range(3)))
            acc0 = tuple(VALUES[rng.integers(0, len(VALUES))] for _ in range(3))
            got = skipping_sum3(acc0, parts)
            for c in range(3):
                want = full_sum(acc0[c], [p[c] for p in parts])
                if np.isnan(want):
                    assert np.isnan(got[c])
                else:
                    assert bits(got[c]) == bits(want)
