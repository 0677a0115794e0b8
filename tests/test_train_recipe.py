"""Host-side pieces of the denoiser's training recipe: the learning-rate schedule and the
weights file (no GPU: a stand-in object supplies and receives the parameters)."""
import numpy as np

from webgpuraytracer_b200 import kpcn
from webgpuraytracer_b200.train_denoiser import parse_schedule


def test_schedule_phases_sum_to_the_steps():
    ph = parse_schedule("0.65:1,0.2:0.3,0.15:0.1", 24000)
    assert ph == [(15600, 1.0), (4800, 0.3), (3600, 0.1)]
    assert sum(n for n, _ in parse_schedule("0.33:1,0.33:0.5,0.34:0.25", 1001)) == 1001
    assert parse_schedule("1:1", 7) == [(7, 1.0)]
    assert parse_schedule("0.5:1,0.5:0.1", 1) == [(1, 1.0)]      # empty phases are dropped


class _Net:
    def __init__(self, p):
        self.p = p

    def get_params(self):
        return self.p

    def set_params(self, a):
        self.p = np.array(a, np.float32)


def test_weights_file_roundtrip(tmp_path):
    src = _Net(np.random.default_rng(1).standard_normal(kpcn.N_PARAMS).astype(np.float32))
    meta = {"family": "flagship", "input_spp": [1, 2, 4], "steps": 10}
    kpcn.save_weights(src, tmp_path / "w.npz", meta)
    dst = _Net(None)
    assert kpcn.load_weights(dst, tmp_path / "w.npz") == meta
    np.testing.assert_array_equal(dst.p, src.p)
