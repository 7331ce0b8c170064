"""Training-pair shards (host side): round trip, order, layout checks."""
import json

import numpy as np
import pytest


def test_pair_shards_round_trip(tmp_path):
    from mpm_snow_sim2d_b200 import mlp_train
    rows = np.random.default_rng(0).standard_normal((2500, 20)).astype(np.float32)
    names = mlp_train.save_pair_shards(rows, tmp_path, shard_rows=1000)
    assert names == ["pairs_00000.npy", "pairs_00001.npy", "pairs_00002.npy"]
    idx = json.loads((tmp_path / "index.json").read_text())
    assert idx["rows"] == 2500 and idx["layout"] == mlp_train.PAIR_LAYOUT
    back = mlp_train.load_pair_shards(tmp_path)
    assert back.dtype == np.float32 and np.array_equal(back, rows)


def test_pair_shards_reject_bad_input(tmp_path):
    from mpm_snow_sim2d_b200 import mlp_train
    with pytest.raises(ValueError):
        mlp_train.save_pair_shards(np.zeros((4, 19), np.float32), tmp_path)
    mlp_train.save_pair_shards(np.zeros((4, 20), np.float32), tmp_path)
    idx = json.loads((tmp_path / "index.json").read_text())
    idx["rows"] = 5
    (tmp_path / "index.json").write_text(json.dumps(idx))
    with pytest.raises(ValueError):
        mlp_train.load_pair_shards(tmp_path)
