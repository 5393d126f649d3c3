"""The bank-conflict model behind the TE kernel's table layout and sample order
(tenex_b200/bank_model.py) on cfg4's generator: the odd row stride costs fewer
wavefronts per reduction than stride b_s, sorting each lane's samples by target
state fewer again, and the magnitudes sit where ncu put the kernel (3.10 with
stride b_s, 2.88 with the odd stride, on a cfg4 slice)."""
import numpy as np

from oracle import oracle as O
from tenex_b200 import bank_model as BM
from tenex_b200 import workloads as W


def test_single_reduction_counts_distinct_words_per_bank():
    assert BM.reduction_wavefronts(np.arange(32)) == 1           # one word per bank
    assert BM.reduction_wavefronts(np.zeros(32, np.int64)) == 1  # one word, merged
    assert BM.reduction_wavefronts(np.arange(32) * 32) == 32     # 32 words in bank 0
    assert BM.reduction_wavefronts(np.array([0, 32, 32, 64] + [1] * 28)) == 3


def test_layout_choices_on_cfg4_bins():
    x, npv = W.cfg4_bins(300, 8193, seed=1004)
    cb, cnpv, _ = O.coarsen(x, npv, 38)
    rng = np.random.default_rng(0)
    light = np.where(cnpv < 38)[0]
    even, odd, srt = [], [], []
    for _ in range(40):
        t, s = rng.choice(light, 2, replace=False)
        bt, bs = int(cnpv[t]), int(cnpv[s])
        z = BM.joint_states(cb[t], bt)
        y = cb[s, :-1]
        even.append(BM.pair_wavefronts(z, y, bs, max_chunks=8))
        odd.append(BM.pair_wavefronts(z, y, bs | 1, max_chunks=8))
        srt.append(BM.pair_wavefronts(z, y, bs | 1, sort_groups=True, max_chunks=8))
    e, o, s = np.mean(even), np.mean(odd), np.mean(srt)
    assert 2.9 < e < 3.4 and 2.6 < o < 3.0 and 2.2 < s < 2.6, (e, o, s)
    assert s < o < e
