"""The named configurations (nebula_b200/configs.json) build the scenes the
bench and the parity tests use, with the stated sizes."""
import json

import numpy as np

from nebula_b200 import scenes as S


def test_every_config_builds_with_its_stated_size():
    cfgs = json.loads(S.CONFIGS_JSON.read_text())["configs"]
    for key, c in cfgs.items():
        if key in ("cfg3", "cfg4"):
            continue  # large: checked below without building the terrain / all 64 scenes twice
        sc = S.load_config(key)
        assert sc.name == c["name"] and sc.n == c["particles"], key


def test_large_configs_match_their_generators():
    cfgs = json.loads(S.CONFIGS_JSON.read_text())["configs"]
    mix = S.load_config("cfg4")
    assert len(mix) == cfgs["cfg4"]["scenes"] and [sc.n for sc in mix] == S.batch_mix_sizes()
    slope = S.load_config("cfg3")
    assert slope.n == cfgs["cfg3"]["particles"] and slope.name == cfgs["cfg3"]["name"]
    ref = S.slope_flow()
    assert np.array_equal(slope.state["P"], ref.state["P"]) and np.array_equal(slope.sdf, ref.sdf)
