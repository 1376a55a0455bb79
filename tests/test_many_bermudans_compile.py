"""Plans with more than 4 Bermudans (beyond the reference kernel's limit): the compiler's term layout -- each
Bermudan's index split over the reference's 4-bit field and the trade-group field, its exercise terms directly
before its policy record -- and the plans it refuses."""
import numpy as np
import pytest

from zlatko_b200 import gpu, workloads
from zlatko_b200 import spec as S


def bermudan_of(code):
    return ((code >> 8) & 15) | (((code >> 4) & 15) << 4)


def test_term_layout_of_twenty_bermudans():
    m, books, _ = workloads.bermudan_book(256, 20)
    ns = S.NettingSet([t for b in books for t in b.trades], None)
    p = gpu.compile(m, ns, S.Options())
    assert int(p.header[27]) == 20
    t = p.terms.reshape(-1, 8)
    codes = t[:, 0].astype(np.int64)
    kinds = codes & 15
    amc = (kinds >= 5) & (kinds <= 9)
    assert set(bermudan_of(codes[amc]).tolist()) == set(range(20))
    for j in range(p.num_dates):
        seen_decide = set()
        for u in range(int(p.indices[j]), int(p.indices[j + 1])):
            k, b = int(kinds[u]), int(bermudan_of(codes[u]))
            if k == 5:
                assert b not in seen_decide  # a Bermudan's exercise terms come before its policy record
            if k == 6:
                seen_decide.add(b)
                assert u > 0 and int(kinds[u - 1]) == 5 and int(bermudan_of(codes[u - 1])) == b
    # Four or fewer keep the reference's layout: no Bermudan bits in the trade-group field.
    p4 = gpu.compile(m, books[0], S.Options())
    c4 = p4.terms.reshape(-1, 8)[:, 0].astype(np.int64)
    assert np.all(((c4 >> 4) & 15) == 0)


def test_refused_plans():
    m, books, _ = workloads.bermudan_book(256, 20)
    ns = S.NettingSet([t for b in books for t in b.trades], None)
    with pytest.raises(ValueError, match="per-trade"):
        gpu.compile(m, ns, S.Options(per_trade=True))
    with pytest.raises(ValueError, match="nested initial margin"):
        gpu.compile(m, S.NettingSet(ns.trades[:6], None), S.Options(im_quantile=0.99, im_inner_paths=64))
