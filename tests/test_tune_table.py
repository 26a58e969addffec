"""The tuner's table handling without a GPU: the committed tuning_table.h
reads back into entries that write the same file, and measured tensor-core
thresholds land on the batched configuration's keys, one per plan type and
window width, leaving every other entry as it was."""

from __future__ import annotations

from pathlib import Path

from wgpunufft_b200 import tune

TABLE = Path(tune.__file__).resolve().parent / "csrc" / "tuning_table.h"


def test_committed_table_reads_back_to_the_same_file():
    entries = tune.read_table(TABLE)
    assert entries, "no entries parsed"
    assert tune.table_header(entries) == TABLE.read_text()
    keys = [tuple(sorted(e["key"].items())) for e in entries]
    assert len(keys) == len(set(keys)), "one entry per key"


def test_tensor_thresholds_merge_per_type_and_width(monkeypatch, tmp_path):
    entries = tune.read_table(TABLE)
    before = {tuple(sorted(e["key"].items())): dict(e) for e in entries}
    widths = {1e-2: 3, 1e-3: 4, 1e-4: 5, 1e-5: 6, 1e-6: 7}
    thresholds = {(1, 3): 16, (2, 3): 256, (1, 4): 16, (2, 4): 256, (1, 5): 32, (2, 5): 128, (1, 6): 16,
                  (2, 6): 64, (1, 7): 16, (2, 7): 0}
    assert tuple(widths) == tune.TENSOR_EPS

    def fake(torch, w, workloads, native, kind, eps, repeats):
        width = widths[eps]
        times = {b: {"tensor_cores": 1.0, "cuda_cores": 2.0} for b in tune.TENSOR_BATCHES}
        return thresholds[(kind, width)], width, times

    monkeypatch.setattr(tune, "tune_tensor_threshold", fake)
    measured = tune.tensor_entries(None, None, None, None, entries, 1)
    assert [(m["type"], m["width"], m["threshold"]) for m in measured] == [
        (kind, width, thresholds[(kind, width)]) for kind in (1, 2) for width in widths.values()]
    by_key = {tuple(sorted(e["key"].items())): e for e in entries}
    assert len(by_key) == len(entries), "one entry per key"
    for (kind, width), threshold in thresholds.items():
        key = {"type": kind, "dimensions": 2, "precision": 3, "width": width, "log2_cells": 20, "log2_density": 0}
        entry = by_key[tuple(sorted(key.items()))]
        assert entry["tensor_min_batch"] == (threshold or 1 << 30)
    # A new key keeps the launch choices the library gave it before: those
    # of the nearest type-1 entry of its width (the 1024^2 entry for w 6).
    w6 = by_key[tuple(sorted({"type": 1, "dimensions": 2, "precision": 3, "width": 6, "log2_cells": 20,
                              "log2_density": 0}.items()))]
    assert (w6["best"]["tile"], w6["best"]["ctas_per_sm"]) == (64, 2)
    # Launch choices of existing keys are kept; other keys are untouched.
    for k, old in before.items():
        new = by_key[k]
        assert new["best"] == old["best"]
        if dict(k)["log2_cells"] != 20 or dict(k)["dimensions"] != 2 or dict(k)["precision"] != 3:
            assert new["tensor_min_batch"] == old["tensor_min_batch"]
    # The written table parses back to the merged entries.
    path = tmp_path / "tuning_table.h"
    path.write_text(tune.table_header(entries))
    assert tune.read_table(path) == entries
