"""Host-side logic of the learned jump (no GPU): the sizes of the fallback
pool, which redoes only the members the judge rejects on a model of about
their count."""
import pytest

from symphas_b200 import surrogate as S


@pytest.mark.parametrize("batch", [1, 2, 7, 64, 256, 1000])
def test_fallback_pool_sizes(batch):
    pool = S.FdPool(256, batch, 0.01)
    sizes = pool.sizes
    assert sizes[0] == 1 and sizes[-1] == batch
    assert all(b > a for a, b in zip(sizes, sizes[1:]))
    # every count of rejected members is padded by at most a quarter (and one)
    for a, b in zip(sizes, sizes[1:]):
        assert b <= max(a + 1, int(a * 1.25 + 0.5)) or b == batch
    assert pool.models == {}  # nothing is created before it is needed
