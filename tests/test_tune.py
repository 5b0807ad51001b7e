"""Tile-configuration table of the autotuner (host side, no GPU): set and
read back per feature shape, rejection of values the kernels do not
support, and the committed table's format."""
import json
import os

import numpy as np
import pytest

from librascal_b200 import _native as N, tune


def test_set_get_remove():
    shape = (3, 5, 4)
    assert tune.get_config(shape) == tune.DEFAULT
    cfg = dict(tune.DEFAULT, exp_chunk=32, exp_warps=8, adj_threads=64, psb_threads=160, gemm_variant=2)
    tune.set_config(shape, cfg)
    assert tune.get_config(shape) == cfg
    assert tune.get_config((3, 5, 5)) == tune.DEFAULT  # other shapes untouched
    tune.set_config(shape, None)
    assert tune.get_config(shape) == tune.DEFAULT


@pytest.mark.parametrize("field,value", [("exp_chunk", 12), ("exp_warps", 0), ("exp_warps", 9),
                                         ("adj_threads", 48), ("adj_threads", 256), ("adj_blocks_per_sm", 0),
                                         ("psf_threads", 512), ("psb_threads", 100), ("gemm_variant", 3)])
def test_rejects_unsupported(field, value):
    with pytest.raises(RuntimeError, match="tile config"):
        tune.set_config((2, 4, 3), dict(tune.DEFAULT, **{field: value}))
    assert tune.get_config((2, 4, 3)) == tune.DEFAULT


def test_every_candidate_is_accepted():
    for field in tune.FIELDS:
        for v in tune.CANDIDATES[field]:
            tune.set_config((1, 2, 1), dict(tune.DEFAULT, **{field: v}))
    tune.set_config((1, 2, 1), None)


def test_committed_table_format():
    if not os.path.exists(tune.TABLE):
        pytest.skip("no tuned table committed")
    d = json.load(open(tune.TABLE))
    assert d["fields"] == tune.FIELDS
    for e in d["entries"]:
        assert len(e["shape"]) == 3
        for f in tune.FIELDS:
            # entries written before a field existed keep its default
            assert e["values"].get(f, tune.DEFAULT[f]) in tune.CANDIDATES[f]
        assert len(e["default_stage_ms"]) == 8 and len(e["tuned_stage_ms"]) == 8
    # the package installed it when it loaded the library
    N.lib()
    for e in d["entries"]:
        assert tune.get_config(e["shape"]) == dict(tune.DEFAULT, **e["values"])
