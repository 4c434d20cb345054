"""The balanced atom-split form's partition of the (point tile, atom) space, restated on the host:
equal contiguous ranges per CTA (to one unit), the inverse map from a unit to its CTA, the stage
count each CTA derives in closed form (the producer and the consumers must agree on it, or the
ring would be refilled past the CTA's range), and the pieces of every split tile (at most two per
CTA, the slot rule of the fix-up).  Mirrors BalanceSplit and the stage rules of
ktt_b200/csrc/coul_forward.cuh (kBalStageAtoms 4096, kBalFirstAtoms 1024)."""
import random

STAGE, FIRST = 4096, 1024


def start(b, q, r):
    return b * q + min(b, r)


def cta_of(u, q, r):
    big = r * (q + 1)
    return u // (q + 1) if u < big else r + (u - big) // q


def walk_stages(tb, ab, te, ast, n):
    """The stage sequence as the kernel walks it: (tile, first atom, count)."""
    out, t, a = [], tb, ab
    while t <= te:
        pe = ast if t == te else n
        cap = FIRST if (t == tb and a == ab) else STAGE
        c = min(pe - a, cap)
        out.append((t, a, c))
        a += c
        if a == pe:
            t, a = t + 1, 0
    return out


def closed_form_stages(tb, ab, te, ast, n):
    so = lambda x: (x + STAGE - 1) // STAGE
    first_len = (ast if tb == te else n) - ab
    return 1 + so(max(0, first_len - FIRST)) + ((te - tb - 1) * so(n) + so(ast) if te > tb else 0)


def check(tiles, n, ctas):
    units = tiles * n
    q, r = divmod(units, ctas)
    assert q >= 1
    pieces = {}
    for b in range(ctas):
        ub, ue = start(b, q, r), start(b + 1, q, r)
        assert ue - ub in (q, q + 1)
        assert cta_of(ub, q, r) == b and cta_of(ue - 1, q, r) == b
        tb, ab = divmod(ub, n)
        te, last = divmod(ue - 1, n)
        ast = last + 1
        stages = walk_stages(tb, ab, te, ast, n)
        assert sum(c for _, _, c in stages) == ue - ub
        assert len(stages) == closed_form_stages(tb, ab, te, ast, n)
        for t in range(tb, te + 1):
            lo = ab if t == tb else 0
            hi = ast if t == te else n
            if lo == 0 and hi == n:
                continue  # whole tile, stored by this CTA
            assert t in (tb, te)  # only a CTA's first and last pieces can be split
            slot = 0 if t == tb else 1
            assert slot == (0 if start(b, q, r) >= t * n else 1)
            pieces.setdefault(t, []).append((b, lo, hi))
    for t, ps in pieces.items():
        first, last = cta_of(t * n, q, r), cta_of((t + 1) * n - 1, q, r)
        assert [b for b, _, _ in ps] == list(range(first, last + 1))
        assert sum(hi - lo for _, lo, hi in ps) == n  # the pieces tile the atoms exactly once


def test_partition_of_the_slice_and_of_a_small_map():
    check(128, 4000, 148)   # the 256 x 256 slice, 32 x 1 tile threads x 16 points
    check(64, 4000, 148)    # the same with 64 x 1 tile threads
    check(4096, 16384, 148)  # 256 x 256 x 64, 1,024-point tiles


def test_partition_of_random_shapes():
    rng = random.Random(5)
    for _ in range(400):
        tiles, n, ctas = rng.randint(1, 300), rng.randint(1, 20000), rng.randint(1, 600)
        if tiles * n < ctas:
            ctas = tiles * n  # the host caps the grid at one unit per CTA
        check(tiles, n, ctas)
