"""dtlg_or_words, the device OR of sharded Bloom builds, against numpy; and a
sharded build on one GPU (world size 1 of the same code) against the full one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

import dtlg as F  # noqa: E402
from dtlg import keygen  # noqa: E402
from dtlg.shard import or_words, shard_bounds  # noqa: E402


@pytest.mark.parametrize("n,parts", [(1, 1), (1000003, 3), (1 << 22, 4)])
def test_or_words_matches_numpy(n, parts):
    rng = np.random.default_rng(n)
    dst = rng.integers(0, 2 ** 63, n, dtype=np.int64)
    src = [rng.integers(0, 2 ** 63, n, dtype=np.int64) for _ in range(parts)]
    d = torch.from_numpy(dst.copy()).cuda()
    or_words(d, [torch.from_numpy(s).cuda() for s in src])
    want = dst.copy()
    for s in src:
        want |= s
    assert np.array_equal(d.cpu().numpy(), want)


def test_partial_builds_or_to_the_full_build():
    cfg = F.blocked_bloomfilter_config(k=8, word_size=8, word_cnt_per_block=8, sector_cnt=8)
    n, world = 1 << 20, 4
    f = F.construct(cfg, n * 12 + 5)
    keys = keygen.build_keys_torch(n, 9)
    parts = []
    for r in range(world):
        a, c = shard_bounds(n, r, world)
        w = f.alloc_filter_data()
        assert f.batch_insert(w, keys[a:a + c].contiguous())
        parts.append(w)
    full = f.alloc_filter_data()
    assert f.batch_insert(full, keys)
    combined = parts[0].clone()
    or_words(combined, parts[1:])
    assert torch.equal(combined, full)
